// pcf_solver.cu -- the C ABI of include/pincflow_poisson.h: handle life cycle,
// uploads, the BiCGSTAB driver (reference FP64 and mixed FP32/FP64) and the
// component entry points.
//
// The Krylov loop follows apply_bicgstab!.jl:24-150 step by step; every
// scalar (alpha, omega, beta, the residual test) lives on the device and is
// computed by the last block of the kernel that produces its dot products, so
// an iteration is a fixed sequence of launches with no host round trip.  The
// host only polls the status word every `check_interval` iterations; kernels
// launched after convergence see the done flag and return at once.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include <cuda.h>

#include "pcf_kernels.cuh"
#include "pcf_mg.cuh"
#include "pcf_tiny.cuh"

namespace {
thread_local cudaError_t g_last_cuda = cudaSuccess;
}

int pcf_set_cuda_error(cudaError_t e) {
    g_last_cuda = e;
    return e == cudaErrorMemoryAllocation ? PCF_ENOMEM : PCF_ECUDA;
}

int pcf_launch_assemble(pcf_handle *h, double dt, double rf, int damp_h, int c0 = 0, int c1 = -1);
int pcf_assemble_chunk_levels();
int pcf_launch_factors(pcf_handle *h, double deta);
int pcf_launch_correct(pcf_handle *h, double dt, double rf, int damp_h, double *dpip, double *u, double *v,
                       double *w, double *rhop, double *pip, double *corx, double *cory);
int pcf_launch_fill_predictands(pcf_handle *h, double *rho, double *rhop, double *u, double *v, double *w,
                                double *pip, double *p);
int pcf_launch_modify_wind(pcf_handle *h, const double *p, double *u, double *v, double *w, int divide);
int pcf_launch_predictor(pcf_handle *h, double dt, double rf, int damp_h, double *u, double *v, double *w,
                         double *rho, double *rhop, double *pip, double *p, const double *betar, const double *dudt,
                         const double *dvdt, double *wold);

namespace pcf {

// --------------------------------------------------------- instrumentation --

struct ProfState {
    std::vector<cudaEvent_t> pool;
    size_t used = 0;
    std::vector<ProfRec> pending;
};

static cudaEvent_t prof_event(pcf_handle *h) {
    ProfState *ps = h->prof;
    if (ps->used == ps->pool.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        ps->pool.push_back(e);
    }
    return ps->pool[ps->used++];
}

// Times one launch when profiling is on; counts it always.
struct ProfScope {
    pcf_handle *h;
    int tag;
    double bytes;
    cudaEvent_t a = nullptr;
    // nlaunch: kernel launches the scope covers (counted here unless the
    // launcher counts them itself, nlaunch = 0)
    ProfScope(pcf_handle *h_, int tag_, double bytes_, int nlaunch = 1) : h(h_), tag(tag_), bytes(bytes_) {
        h->launches += nlaunch;
        if (h->prof_on && h->prof) {
            a = prof_event(h);
            if (a) cudaEventRecord(a, h->stream);
        }
    }
    ~ProfScope() {
        if (a) {
            cudaEvent_t b = prof_event(h);
            if (b) {
                cudaEventRecord(b, h->stream);
                h->prof->pending.push_back({a, b, tag, h->prof_iter, bytes});
            }
        }
    }
};

// Accumulates the pending records (after a stream synchronisation); records
// of iterations >= keep_below (launched after convergence) are dropped.
static void prof_flush(pcf_handle *h, int keep_below) {
    ProfState *ps = h->prof;
    if (!ps) return;
    if (!ps->pending.empty()) {
        cudaStreamSynchronize(h->stream);
        for (const ProfRec &r : ps->pending) {
            if (r.iter >= 0 && r.iter >= keep_below) continue;
            float ms = 0;
            if (cudaEventElapsedTime(&ms, r.a, r.b) != cudaSuccess) continue;
            ProfAcc &acc = h->prof_acc[r.tag];
            acc.ms += ms;
            acc.count += 1;
            acc.bytes += r.bytes;
        }
    }
    ps->pending.clear();
    ps->used = 0;
}

// ------------------------------------------------------------ launchers --

static int num_sms() {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

static ReduceCtx red(pcf_handle *h, KrylovScalars *scal, int op, double *out = nullptr) {
    ReduceCtx c;
    c.partials = h->partials;
    c.ticket = h->ticket;
    c.scal = scal;
    c.out = out;
    c.op = op;
    return c;
}

// Levels per block: enough z-chunks for ~8 blocks per SM, at most
// kMaxPartials blocks.  Each chunk re-reads 4 halo planes of s, so chunks
// are kept at 4 levels or more (only grids too small to fill the GPU, such
// as coarse multigrid levels, get that short).
static int pick_kc(long long xyblocks, int nz) {
    const long long want = 8LL * num_sms();
    long long chunks = (want + xyblocks - 1) / xyblocks;
    if (chunks < 1) chunks = 1;
    long long kc = (nz + chunks - 1) / chunks;
    // at least 4 levels per block amortise the 5-plane prologue on large
    // grids; grids of a few x-y tiles (coarse multigrid levels, L2-resident)
    // are latency-bound, and one level per block shortens each block's chain
    const long long kmin = xyblocks >= 16 ? 4 : 1;
    if (kc < kmin) kc = kmin;
    if (kc > nz) kc = nz;
    while (kc < nz && xyblocks * ((nz + kc - 1) / kc) > kMaxPartials) kc = std::min<long long>(2 * kc, nz);
    return (int)kc;
}

// dynamic shared memory of the staged stencil (C16 = 2: BF16 planes, 3:
// FP8): the stages, one mbarrier each
template <int V, int TX, int TY, bool HORIZ, int C16 = 2>
constexpr int stencil_bulk_smem() {
    return kStencilStages * (stencil_stage_bytes<V, TX, TY, HORIZ, C16 == 3 ? 1 : 2>() + (int)sizeof(uint64_t));
}

// The tensor maps of a BF16 operator copy (25 planes of nx x ny x nz values)
// that the staged stencils load their tiles with, written to the device
// array maps (6 x 128 bytes): boxes of 128 x 4 x 1 values of [0] all 25
// planes, [1] the 4 planes AL..AF, [2] the 18 planes ALD..AFUU, then [3..5]
// the same with 64-wide boxes.  Returns false (and the stencils read the
// planes directly) when the driver has no tensor-map encoder or the grid
// breaks the copy's alignment rules (x rows of a multiple of 16 bytes, at
// least one 128-wide box wide).
static bool make_coef16_maps(const __nv_bfloat16 *coef16, const Dims &d, void *maps) {
    using Encode = decltype(&cuTensorMapEncodeTiled);
    static Encode encode = [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            fn = nullptr;
        }
        return reinterpret_cast<Encode>(fn);
    }();
    if (!encode || !coef16 || d.nx % 8 != 0 || d.nx < 128 || (reinterpret_cast<uintptr_t>(coef16) & 15) != 0)
        return false;
    CUtensorMap host[6];
    const cuuint64_t dims[4] = {(cuuint64_t)d.nx, (cuuint64_t)d.ny, (cuuint64_t)d.nz, (cuuint64_t)PCF_NCOEF};
    const cuuint64_t strides[3] = {2ull * d.nx, 2ull * d.plane, 2ull * (cuuint64_t)d.n};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const cuuint32_t planes[3] = {PCF_NCOEF, PCF_AD - PCF_AL, PCF_NCOEF - PCF_ALD};
    for (int q = 0; q < 6; ++q) {
        const cuuint32_t box[4] = {q < 3 ? 128u : 64u, 4, 1, planes[q % 3]};
        if (encode(&host[q], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16 *>(coef16), dims, strides,
                   box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    }
    return cudaMemcpy(maps, host, sizeof(host), cudaMemcpyHostToDevice) == cudaSuccess;
}

// The tensor maps of an FP8 operator copy (25 planes of nx x ny x nz bytes)
// for the staged pseudo-time step, written to the device array maps (4 x 128
// bytes): boxes of 128 x 4 x 1 values of [0] the 4 planes AL..AF and [1] the
// 18 planes ALD..AFUU, then [2..3] the same with 64-wide boxes.  False when
// the grid breaks the alignment rules (rows of a multiple of 16 bytes, at
// least one 128-wide box wide) or no encoder is available.
static bool make_coef8_maps(const uint8_t *coef8, const Dims &d, void *maps) {
    using Encode = decltype(&cuTensorMapEncodeTiled);
    static Encode encode = [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            fn = nullptr;
        }
        return reinterpret_cast<Encode>(fn);
    }();
    if (!encode || !coef8 || d.nx % 16 != 0 || d.nx < 128 || (reinterpret_cast<uintptr_t>(coef8) & 15) != 0)
        return false;
    CUtensorMap host[4];
    const cuuint64_t dims[4] = {(cuuint64_t)d.nx, (cuuint64_t)d.ny, (cuuint64_t)d.nz, (cuuint64_t)PCF_NCOEF};
    const cuuint64_t strides[3] = {(cuuint64_t)d.nx, (cuuint64_t)d.plane, (cuuint64_t)d.n};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const cuuint32_t planes[2] = {PCF_AD - PCF_AL, PCF_NCOEF - PCF_ALD};
    for (int q = 0; q < 4; ++q) {
        const cuuint32_t box[4] = {q < 2 ? 128u : 64u, 4, 1, planes[q % 2]};
        if (encode(&host[q], CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, const_cast<uint8_t *>(coef8), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    }
    return cudaMemcpy(maps, host, sizeof(host), cudaMemcpyHostToDevice) == cudaSuccess;
}

// Raises the staged stencil's dynamic shared-memory limit on the current
// device (once per device) and returns how many of its blocks the device
// holds at once (resident blocks per SM x SMs); 0 if the device refuses.
template <typename T, int V, int TX, int TY, bool HORIZ, int EPI, bool DIFF, int C16 = 2>
static int stencil_bulk_ready() {
    static std::atomic<int> state[64];  // per device: 0 unknown, -1 refused, else the capacity
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return 0;
    }
    int st = state[dev].load();
    if (st == 0) {
        auto kern = k_stencil<T, V, TX, TY, HORIZ, EPI, DIFF, C16>;
        constexpr int smem = stencil_bulk_smem<V, TX, TY, HORIZ, C16>();
        int per_sm = 0;
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TX * TY, smem) == cudaSuccess &&
            per_sm > 0) {
            st = per_sm * num_sms();
        } else {
            cudaGetLastError();
            st = -1;
        }
        state[dev].store(st);
    }
    return st > 0 ? st : 0;
}

// Launches the TMA-staged stencil (C16 = 2: BF16 planes, 3: FP8) with SV x
// values per thread (tiles of 32 SV x 4 cells) on the handle's stream; false
// (nothing launched) if the device refuses its shared memory or the grid
// exceeds the partials buffer.
template <typename T, int SV, bool HORIZ, int EPI, bool DIFF, int C16 = 2>
static bool launch_staged(pcf_handle *h, const StencilArgs<T> &a0) {
    StencilArgs<T> a = a0;
    if (h->test_stall) a.stall_level = h->test_stall - 1;
    if (h->test_wait_ns) a.wait_ns = h->test_wait_ns;
    const int cap = stencil_bulk_ready<T, SV, 32, 4, HORIZ, EPI, DIFF, C16>();
    if (cap <= 0) return false;
    constexpr int W = 32 * SV;
    const long long gx = (a.nx + W - 1) / W, gy = (a.ny + 3) / 4, xy = gx * gy;
    if (gy > 65535) return false;
    // z-chunks of pick_kc's length, or a half or a quarter of it when that
    // fills the last wave of resident blocks better (measured at
    // 512x512x192 with 128-wide tiles: 1536 blocks in 444 slots, 3.46 waves,
    // 606 us; 3072 blocks, 6.92 waves, 563 us)
    auto fill = [&](int kcx) {
        const long long blocks = xy * ((a.nz + kcx - 1) / kcx);
        return (double)blocks / (double)(((blocks + cap - 1) / cap) * cap);
    };
    int kc = std::min(pick_kc(xy, a.nz), a.nz);
    for (int halvings = 0; halvings < 2; ++halvings) {
        const int c = std::max(1, (kc + 1) / 2);
        if (c == kc || xy * ((a.nz + c - 1) / c) > kMaxPartials || !(fill(c) > fill(kc) + 0.02)) break;
        kc = c;
    }
    const long long gz = (a.nz + kc - 1) / kc;
    if (xy * gz > kMaxPartials) return false;
    k_stencil<T, SV, 32, 4, HORIZ, EPI, DIFF, C16><<<dim3((unsigned)gx, (unsigned)gy, (unsigned)gz), dim3(32, 4, 1),
                                                       stencil_bulk_smem<SV, 32, 4, HORIZ, C16>(), h->stream>>>(a, kc);
    return true;
}

template <typename T, int V, int TX, bool HORIZ, int EPI, bool DIFF>
static int launch_stencil_cfg(pcf_handle *h, const StencilArgs<T> &a, int tag_override, int kc) {
    constexpr int TY = 128 / TX;
    constexpr int W = TX * V;
    const long long gx = (a.nx + W - 1) / W, gy = (a.ny + TY - 1) / TY;
    if (kc <= 0) kc = pick_kc(gx * gy, a.nz);
    kc = std::min(kc, a.nz);
    // one partial sum per block: the grid must fit the partials buffer
    if (gx * gy * ((a.nz + kc - 1) / kc) > kMaxPartials || gy > 65535) return PCF_ERANGE;
    const dim3 grid((unsigned)gx, (unsigned)gy, (unsigned)((a.nz + kc - 1) / kc));
    const dim3 block(TX, TY, 1);
    // algorithmic words per cell: coefficient planes + input + output (+ second operand)
    const int planes = HORIZ ? 22 : 25;
    const int words = planes + 2 + (EPI == EPI_STORE ? 0 : 1);
    const int tag = tag_override >= 0 ? tag_override
                    : a.guard_update ? PCF_PROF_RELIABLE
                    : HORIZ          ? (sizeof(T) == 4 ? PCF_PROF_PSEUDO32 : PCF_PROF_PSEUDO64)
                                     : (sizeof(T) == 4 ? PCF_PROF_APPLY32 : PCF_PROF_APPLY64);
    // the preconditioner's stencils may read BF16 planes (a.coef16)
    constexpr bool c16_ok = sizeof(T) == 4 && !DIFF && (EPI == EPI_PSEUDO || EPI == EPI_RESNR);
    if constexpr (c16_ok && HORIZ && EPI == EPI_PSEUDO && V == 4 && TX == 32) {
        // the finest level's pseudo-time step on the FP8 copy of its planes
        if (a.tmap8 && a.inv8) {
            ProfScope ps(h, tag_override >= 0 ? tag_override : PCF_PROF_MG_BF16,
                         ((double)planes + (double)(words - planes) * sizeof(T)) * (double)a.n);
            const bool narrow = a.n >= 10000000 || a.nx >= 512 || (a.nx % 128 != 0 && a.nx % 64 == 0);
            if (narrow ? launch_staged<T, 2, HORIZ, EPI, DIFF, 3>(h, a) : launch_staged<T, 4, HORIZ, EPI, DIFF, 3>(h, a)) {
                PCF_CUDA_TRY(cudaGetLastError());
                return PCF_OK;
            }
        }
    }
    if constexpr (c16_ok) {
        if (a.coef16) {
            ProfScope ps(h, tag_override >= 0 ? tag_override : PCF_PROF_MG_BF16,
                         ((double)planes * 2 + (double)(words - planes) * sizeof(T)) * (double)a.n);
            // half the bytes per level: a quarter of the levels per block keeps
            // enough loads in flight (measured 137 -> 124 us at 256x256x128,
            // 721 -> 599 us at 512x512x192; an eighth is slower again)
            int kc16 = std::max(1, (kc + 3) / 4);
            if (gx * gy * ((a.nz + kc16 - 1) / kc16) > kMaxPartials) kc16 = kc;  // the grid shape checked above
            const long long gz16 = (a.nz + kc16 - 1) / kc16;
            if constexpr (V == 4 && TX == 32) {
                // the coefficient tiles staged in shared memory by TMA: 64-wide
                // tiles (6 blocks per SM) on grids of 10 million cells or more
                // or rows of 512 or more, 128-wide (3 per SM) otherwise
                // (measured per launch: 512x512x192 0.512 vs 0.561 ms, and the
                // 256x256x192 level below it faster too; 256x256x128 0.116 vs
                // 0.113 ms)
                // (and 64-wide where 128-wide tiles would leave a half-empty
                // column of tiles, nx = 192 for instance)
                const bool narrow = a.n >= 10000000 || a.nx >= 512 || (a.nx % 128 != 0 && a.nx % 64 == 0);
                if (a.tmap16 && (narrow ? launch_staged<T, 2, HORIZ, EPI, DIFF>(h, a)
                                        : launch_staged<T, 4, HORIZ, EPI, DIFF>(h, a))) {
                    PCF_CUDA_TRY(cudaGetLastError());
                    return PCF_OK;
                }
            }
            k_stencil<T, V, TX, TY, HORIZ, EPI, DIFF, 1>
                <<<dim3((unsigned)gx, (unsigned)gy, (unsigned)gz16), block, 0, h->stream>>>(a, kc16);
            PCF_CUDA_TRY(cudaGetLastError());
            return PCF_OK;
        }
    }
    // a guarded reliable-update launch returns at once unless an update is
    // pending; its bytes are counted per update performed (reliable_bytes)
    ProfScope ps(h, tag, a.guard_update ? 0.0 : (double)words * sizeof(T) * (double)a.n);
    k_stencil<T, V, TX, TY, HORIZ, EPI, DIFF><<<grid, block, 0, h->stream>>>(a, kc);
    PCF_CUDA_TRY(cudaGetLastError());
    return PCF_OK;
}

// ------------------------------------------------------------ autotuner --
// Tile shapes of k_stencil: 128 threads as TX x (128 / TX), each thread
// holding V consecutive x values (V = 4 in FP32, 2 in FP64 when nx allows),
// and kc z-levels per block.  The heuristic picks TX = 32 for wide grids and
// TX = 8 otherwise, with pick_kc; with pcf_params.autotune the first solve on
// a grid size times every tile shape at several kc around pick_kc's and keeps
// the fastest for that size class in a process-wide table (per device and
// kernel family), which later launches of any handle consult.
constexpr int kTileX[3] = {32, 16, 8};

static int tune_family(int tsize, bool horiz, bool diff) {
    if (tsize == 8) return horiz ? PCF_TUNE_HORIZ64 : PCF_TUNE_TOTAL64;
    return horiz ? PCF_TUNE_HORIZ32 : diff ? PCF_TUNE_TOTAL32_DIFF : PCF_TUNE_TOTAL32;
}

struct TuneRec {
    int device;
    pcf_tune_entry e;
    int tile;
};
static std::mutex g_tune_mu;
static std::vector<TuneRec> g_tune;

static bool tune_lookup(int family, int device, const Dims &d, int *tile, int *kc) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (const TuneRec &r : g_tune)
        if (r.device == device && r.e.kernel == family && r.e.nx == d.nx && r.e.ny == d.ny && r.e.nz == d.nz) {
            *tile = r.tile;
            *kc = r.e.levels;
            return true;
        }
    return false;
}

static int default_tile(int nx, int vmax) {
    const bool vec = nx % vmax == 0;
    return nx >= (vec ? 32 * vmax : 32) ? 0 : 2;
}

template <typename T, bool HORIZ, int EPI, bool DIFF>
static int launch_tile(pcf_handle *h, const StencilArgs<T> &a, int tile, int kc, int tag) {
    constexpr int VMAX = sizeof(T) == 4 ? 4 : 2;
    const bool vec = (a.nx % VMAX) == 0;
    switch (tile) {
        case 0:
            return vec ? launch_stencil_cfg<T, VMAX, 32, HORIZ, EPI, DIFF>(h, a, tag, kc)
                       : launch_stencil_cfg<T, 1, 32, HORIZ, EPI, DIFF>(h, a, tag, kc);
        case 1:
            return vec ? launch_stencil_cfg<T, VMAX, 16, HORIZ, EPI, DIFF>(h, a, tag, kc)
                       : launch_stencil_cfg<T, 1, 16, HORIZ, EPI, DIFF>(h, a, tag, kc);
        default:
            return vec ? launch_stencil_cfg<T, VMAX, 8, HORIZ, EPI, DIFF>(h, a, tag, kc)
                       : launch_stencil_cfg<T, 1, 8, HORIZ, EPI, DIFF>(h, a, tag, kc);
    }
}

// Stencil apply on a grid of dimensions d (the handle's grid or a multigrid level).
template <typename T, bool HORIZ, int EPI, bool DIFF = false>
static int launch_stencil_dims(pcf_handle *h, StencilArgs<T> a, const Dims &d, int tag = -1) {
    a.nx = d.nx;
    a.ny = d.ny;
    a.nz = d.nz;
    a.n = d.n;
    constexpr int VMAX = sizeof(T) == 4 ? 4 : 2;
    int tile = 0, kc = 0;
    if (!tune_lookup(tune_family(sizeof(T), HORIZ, DIFF), h->dims.device, d, &tile, &kc)) {
        tile = default_tile(a.nx, VMAX);
        kc = 0;
    }
    return launch_tile<T, HORIZ, EPI, DIFF>(h, a, tile, kc, tag);
}

// Times the candidate tile shapes of one kernel family on grid d (once per
// size class and device) with the given operator and scratch vectors.
template <typename T, bool HORIZ, bool DIFF>
static int tune_stencil(pcf_handle *h, const Dims &d, const T *coef, const T *sv, T *out, const T *b) {
    const int family = tune_family(sizeof(T), HORIZ, DIFF);
    int t0, k0;
    if (tune_lookup(family, h->dims.device, d, &t0, &k0)) return PCF_OK;
    constexpr int VMAX = sizeof(T) == 4 ? 4 : 2;
    constexpr int EPI = HORIZ ? EPI_PSEUDO : EPI_STORE;
    StencilArgs<T> a;
    a.coef = coef;
    a.s = sv;
    a.out = out;
    a.w1 = b;
    a.deta = 0.1;
    a.nx = d.nx;
    a.ny = d.ny;
    a.nz = d.nz;
    a.n = d.n;
    const int vmax_ok = d.nx % VMAX == 0 ? VMAX : 1;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    PCF_CUDA_TRY(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return PCF_ECUDA;
    }
    const int saved_prof = h->prof_on;
    h->prof_on = 0;
    // mean time of reps back-to-back launches
    auto trial = [&](int tile, int kc, int reps, double *ms) -> int {
        int rc;
        PCF_CUDA_TRY(cudaEventRecord(e0, h->stream));
        for (int q = 0; q < reps; ++q)
            if ((rc = launch_tile<T, HORIZ, EPI, DIFF>(h, a, tile, kc, -1))) return rc;
        PCF_CUDA_TRY(cudaEventRecord(e1, h->stream));
        PCF_CUDA_TRY(cudaEventSynchronize(e1));
        float f = 0;
        PCF_CUDA_TRY(cudaEventElapsedTime(&f, e0, e1));
        *ms = f / reps;
        return PCF_OK;
    };
    // a warm-up launch, an estimate, then the better of two trials of at
    // least ~0.3 ms each: small grids' 10-us launches timed 3 at a time were
    // noisy enough to pick different tiles from run to run
    auto time_cfg = [&](int tile, int kc, double *ms) -> int {
        int rc = launch_tile<T, HORIZ, EPI, DIFF>(h, a, tile, kc, -1);
        if (rc) return rc;
        double est = 0, t1 = 0, t2 = 0;
        if ((rc = trial(tile, kc, 3, &est))) return rc;
        const int reps = std::max(3, std::min(64, (int)std::ceil(0.3 / std::max(est, 1e-3))));
        if ((rc = trial(tile, kc, reps, &t1)) || (rc = trial(tile, kc, reps, &t2))) return rc;
        *ms = std::min(t1, t2);
        return PCF_OK;
    };
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    const int tdef = default_tile(d.nx, VMAX);
    int best_tile = tdef, best_kc = 0;
    double best = 1e300, def_ms = 0;
    int rc = PCF_OK;
    for (int tile = 0; tile < 3 && rc == PCF_OK; ++tile) {
        const int W = kTileX[tile] * vmax_ok, TY = 128 / kTileX[tile];
        const long long xyb = (long long)((d.nx + W - 1) / W) * ((d.ny + TY - 1) / TY);
        const int kd = pick_kc(xyb, d.nz);
        const int cands[4] = {kd, kd / 2, 2 * kd, 4 * kd};
        for (int q = 0; q < 4 && rc == PCF_OK; ++q) {
            const int kc = std::min(cands[q], d.nz);
            if (kc < 2 || xyb * ((d.nz + kc - 1) / kc) > kMaxPartials) continue;
            bool seen = false;
            for (int r = 0; r < q; ++r) seen |= std::min(cands[r], d.nz) == kc;
            if (seen) continue;
            double ms = 0;
            rc = time_cfg(tile, kc, &ms);
            if (rc) break;
            if (tile == tdef && q == 0) def_ms = ms;
            if (ms < best) {
                best = ms;
                best_tile = tile;
                best_kc = kc;
            }
        }
    }
    h->prof_on = saved_prof;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    TuneRec r;
    r.device = h->dims.device;
    r.tile = best_tile;
    r.e.kernel = family;
    r.e.nx = d.nx;
    r.e.ny = d.ny;
    r.e.nz = d.nz;
    r.e.tile_x = kTileX[best_tile];
    r.e.vec = vmax_ok;
    r.e.levels = best_kc;
    r.e.ms_best = best;
    r.e.ms_default = def_ms;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune.push_back(r);
    return PCF_OK;
}

template <typename T, bool HORIZ, int EPI, bool DIFF = false>
static int launch_stencil(pcf_handle *h, StencilArgs<T> a) {
    return launch_stencil_dims<T, HORIZ, EPI, DIFF>(h, a, h->d);
}

// Total apply of the Krylov loop: plain form, or the FP32 difference form.
template <typename T, int EPI>
static int apply_total(pcf_handle *h, const StencilArgs<T> &a, bool diff) {
    if constexpr (sizeof(T) == 4) {
        if (diff) return launch_stencil<T, false, EPI, true>(h, a);
    }
    return launch_stencil<T, false, EPI>(h, a);
}

template <typename T, int MODE>
static int launch_thomas(pcf_handle *h, const ThomasArgs<T> &a, int tag = -1) {
    const int bs = 128;
    // input forming + P, M (forward) + y write, y read, Q, solution write
    const int words = (MODE == TH_B || MODE == TH_T ? 1 : (MODE == TH_SUPD ? 3 : 4)) + 6;
    ProfScope ps(h, tag >= 0 ? tag : sizeof(T) == 4 ? PCF_PROF_THOMAS32 : PCF_PROF_THOMAS64,
                 (double)words * sizeof(T) * (double)a.n);
    k_thomas<T, MODE><<<(a.plane + bs - 1) / bs, bs, 0, h->stream>>>(a);
    PCF_CUDA_TRY(cudaGetLastError());
    return PCF_OK;
}

static unsigned vec_grid(long long n) {
    long long g = (n + 255) / 256;
    const long long cap = 4LL * num_sms();
    return (unsigned)(g < cap ? (g < 1 ? 1 : g) : cap);
}

// --------------------------------------------------------- precision views --

template <typename T>
struct Work {
    const T *coef, *fac;
    T *x, *r, *r0, *p, *v, *s, *t, *za, *zb, *zc, *zd;  // (za, zb): M p chain, (zc, zd): M s chain
    KrylovScalars *scal;
    const T *coefT;  // planes of the Total apply inside the loop
    const T *post;   // 1 / fcscal when the loop variable is pi = s / fcscal
};

static Work<double> work64(pcf_handle *h) {
    // the reference form consumes M p before M s is formed: one chain suffices
    return {h->coef64, h->fac64, h->x64, h->r64, h->r064, h->p64, h->v64, h->s64, h->t64, h->za64, h->zb64,
            h->za64, h->zb64, h->scal64, h->coef64, nullptr};
}
static Work<float> work32(pcf_handle *h) {
    return {h->coef32, h->fac32, h->x32, h->r32, h->r032, h->p32, h->v32, h->s32, h->t32, h->za32, h->zb32,
            h->zc32, h->zd32, h->scal32, h->coef32, nullptr};
}
// The FP32 loop of the mixed solve: difference-form operator on pi = s / fcscal.
static Work<float> work32_pi(pcf_handle *h) {
    Work<float> w = work32(h);
    w.coefT = h->coefB32;
    w.post = h->rfc32;
    return w;
}

static double deta_of(const pcf_handle *h, double dtau) {
    // apply_preconditioner!.jl:58
    return dtau / (2 * (1 / (h->dx * h->dx) + 1 / (h->dy * h->dy)));
}

// Difference-form FP32 operator (k_build_diff) from the FP64 operator; the
// variable is pi = s / fcscal, with fcscal = 1 when no background is set.
// fcscal on the haloed grid from the background (or 1 without one); the
// assembly and the difference form read it.
static int fcscal_halo(pcf_handle *h, int have_background) {
    h->launches += 1;
    k_fcscal_halo<<<vec_grid(h->nh), 256, 0, h->stream>>>(h->pbar, h->rhobar, h->fch, h->rfch, h->nh,
                                                           have_background);
    PCF_CUDA_TRY(cudaGetLastError());
    return PCF_OK;
}

static int build_diff(pcf_handle *h, int have_background) {
    // with a background, fch was computed when it was set
    if (!have_background) {
        int rc = fcscal_halo(h, 0);
        if (rc) return rc;
    }
    h->launches += 1;
    k_build_diff<<<(unsigned)((h->d.n + 127) / 128), 128, 0, h->stream>>>(
        h->coef64, h->fch, h->d.nx, h->d.ny, h->d.nz, h->dims.nbx, h->dims.nby, h->dims.nbz, h->nxx, h->nyy,
        h->coefB32, h->fc64, h->rfc32);
    PCF_CUDA_TRY(cudaGetLastError());
    return PCF_OK;
}

static int ensure_factors(pcf_handle *h, double deta) {
    if (h->fac_deta == deta) return PCF_OK;
    // ac, ad, au read; P, M, Q written in FP64 and FP32
    ProfScope ps(h, PCF_PROF_ASSEMBLE, (3.0 * 8 + 3.0 * 12) * (double)h->d.n);
    return pcf_launch_factors(h, deta);
}

// M(b) with `iters` pseudo-time steps (apply_preconditioner!.jl:53-121).  The
// first step's Thomas input is formed by MODE (b itself, or the BiCGSTAB
// s / p update, written back to bvec).  Returns the buffer that holds M b.
template <typename T, int MODE>
static int precond_apply(pcf_handle *h, const Work<T> &w, T *bvec, int iters, double deta,
                         const KrylovScalars *guard, T **result, T *o1 = nullptr, T *o2 = nullptr,
                         const T *post = nullptr) {
    if (!o1) {
        o1 = w.za;
        o2 = w.zb;
    }
    ThomasArgs<T> ta;
    ta.fac = w.fac;
    ta.in = bvec;
    ta.r = w.r;
    ta.v = w.v;
    ta.vec = bvec;
    ta.out = o1;
    ta.plane = h->d.plane;
    ta.nz = h->d.nz;
    ta.n = h->d.n;
    ta.deta = deta;
    ta.scal = guard;
    ta.post = iters == 1 ? post : nullptr;  // the last pseudo-time step returns M b / fcscal
    int rc = launch_thomas<T, MODE>(h, ta);
    if (rc) return rc;
    T *cur = o1, *other = o2;
    for (int m = 1; m < iters; ++m) {
        StencilArgs<T> sa;
        sa.coef = w.coef;
        sa.s = cur;
        sa.out = other;
        sa.w1 = bvec;
        sa.deta = deta;
        sa.guard = guard;
        rc = launch_stencil<T, true, EPI_PSEUDO>(h, sa);
        if (rc) return rc;
        ThomasArgs<T> tb = ta;
        tb.in = other;
        tb.out = other;
        tb.post = m == iters - 1 ? post : nullptr;
        rc = launch_thomas<T, TH_T>(h, tb);
        if (rc) return rc;
        T *tmp = cur;
        cur = other;
        other = tmp;
    }
    *result = cur;
    return PCF_OK;
}

// ------------------------------------------------------------ multigrid --
// Horizontal aggregation multigrid V-cycle (pcf_mg.cuh) around the
// reference line relaxation, FP32, used as the right preconditioner of the
// mixed-precision solve.  One cycle on level l with right-hand side b:
//   s = S(b)              one pseudo-time step from zero (vertical Thomas)
//   r = b - A s           restricted to level l+1 and cycled there
//   s += P e              coarse correction
//   s = S(b; s)           one pseudo-time step from s
// and mg_coarse_iterations pseudo-time steps on the coarsest level.

struct MgLevel {
    Dims d;
    int cx = 1, cy = 1;  // aggregation from the finer level (levels >= 1)
    double dx = 0, dy = 0, deta = 0;
    float *coef = nullptr, *fac = nullptr, *fc = nullptr, *b = nullptr, *s = nullptr, *t = nullptr;
    __nv_bfloat16 *coef16 = nullptr;  // level 1: BF16 copy of coef (multigrid BF16 mode)
    void *tmap16 = nullptr;           // levels 0 and 1: tensor maps of the BF16 copy (make_coef16_maps), or null
    void *tmap8 = nullptr;            // level 0: tensor maps of the FP8 copy (make_coef8_maps) while it is used
};
struct MgState {
    std::vector<MgLevel> lv;  // lv[0] is the handle's grid (its planes are the handle's)
    std::vector<void *> allocs;
    int min_columns = -1;
    int coarse_iters = 0;
    long long version = -1;  // operator version the coarse operators were built from
    double dtau = 0;
    bool bf16 = false;       // the finest level's stencils read h->coef16
    void *maps8 = nullptr;   // the FP8 copy's tensor maps (made once)
    int fused_from = -1;     // first level of the one-launch coarse cycle (k_mg_coarse), -1: none
    int coarse_cluster = 0;  // its cluster's CTAs (16, or 8 where 16 is refused)
};

__global__ void k_to_float(const double *__restrict__ a, float *__restrict__ b, long long n, double scale);

// ---- the FP8 copy of the finest level's planes (the pseudo-time step's) ----
// Plane p is stored as E4M3(c16 * scale_p) with scale_p = 2^(7 - e_p), where
// max |c16| over the plane is f 2^e_p (f in [0.5, 1)): the plane's largest
// value lands in [64, 128), below E4M3's 448, and values under 2^-16 of it
// flush to zero.  Scales are powers of 2, so scaling and unscaling are exact.

// max |value| of each of the 25 BF16 planes (blockIdx.y) as the bits of a
// non-negative float, atomically combined into amax (zero beforehand)
__global__ void __launch_bounds__(256) k_plane_absmax(const __nv_bfloat16 *__restrict__ c, long long n,
                                                      unsigned *amax) {
    const __nv_bfloat16 *pl = c + (long long)blockIdx.y * n;
    float m = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(__bfloat162float(pl[i])));
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
    __shared__ float wmax[8];
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmaxf(m, wmax[w]);
        atomicMax(amax + blockIdx.y, __float_as_uint(m));
    }
}

// scale[p] and 1 / scale[p] (at scale + 25) from the planes' maxima
__global__ void k_fp8_scales(const unsigned *amax, float *scale) {
    const int p = threadIdx.x;
    if (p >= PCF_NCOEF) return;
    const float m = __uint_as_float(amax[p]);
    int e = 0;
    if (m > 0.f) frexpf(m, &e);
    scale[p] = m > 0.f ? ldexpf(1.f, 7 - e) : 1.f;
    scale[PCF_NCOEF + p] = m > 0.f ? ldexpf(1.f, e - 7) : 1.f;
}

// c8 = E4M3(c16 * scale) (round to nearest even, saturating), two values per thread
__global__ void __launch_bounds__(256) k_to_fp8(const __nv_bfloat16 *__restrict__ c, long long n,
                                                const float *__restrict__ scale, uint8_t *__restrict__ c8) {
    const float sc = scale[blockIdx.y];
    const __nv_bfloat162 *src = reinterpret_cast<const __nv_bfloat162 *>(c + (long long)blockIdx.y * n);
    __nv_fp8x2_storage_t *dst = reinterpret_cast<__nv_fp8x2_storage_t *>(c8 + (long long)blockIdx.y * n);
    const long long n2 = n / 2;  // n is even (nx % 16 == 0)
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n2; i += (long long)gridDim.x * blockDim.x) {
        float2 v = __bfloat1622float2(src[i]);
        v.x *= sc;
        v.y *= sc;
        dst[i] = __nv_cvt_float2_to_fp8x2(v, __NV_SATFINITE, __NV_E4M3);
    }
}

__global__ void k_float_to_bf16(const float *__restrict__ a, __nv_bfloat16 *__restrict__ b, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = __float2bfloat16_rn(a[i]);
}

// Coarse levels with few columns: k_thomas_split (runs of at most 8 levels,
// up to 32 threads per column); otherwise the column-per-thread sweep.
constexpr int kSplitThomasColumns = 16384;

template <int MODE>
static int mg_thomas(pcf_handle *h, const MgLevel &L, const ThomasArgs<float> &a, int tag) {
    int lpc = 1;
    while (lpc < 32 && (a.nz + lpc - 1) / lpc > 8) lpc *= 2;
    if (L.d.plane > kSplitThomasColumns || (a.nz + lpc - 1) / lpc > 8 || a.post != nullptr || lpc < 2)
        return launch_thomas<float, MODE>(h, a, tag);
    ProfScope ps(h, tag, 6.0 * 4 * (double)a.n);
    const unsigned grid = (unsigned)((a.plane + 31) / 32);
    switch (lpc) {
        case 2: k_thomas_split<MODE, 2><<<grid, dim3(32, 2), 0, h->stream>>>(a); break;
        case 4: k_thomas_split<MODE, 4><<<grid, dim3(32, 4), 0, h->stream>>>(a); break;
        case 8: k_thomas_split<MODE, 8><<<grid, dim3(32, 8), 0, h->stream>>>(a); break;
        case 16: k_thomas_split<MODE, 16><<<grid, dim3(32, 16), 0, h->stream>>>(a); break;
        default: k_thomas_split<MODE, 32><<<grid, dim3(32, 32), 0, h->stream>>>(a); break;
    }
    PCF_CUDA_TRY(cudaGetLastError());
    return PCF_OK;
}

static ThomasArgs<float> mg_targs(const MgLevel &L, const float *fac, const float *in, float *out,
                                  const KrylovScalars *guard) {
    ThomasArgs<float> ta;
    ta.fac = fac;
    ta.in = in;
    ta.r = nullptr;
    ta.v = nullptr;
    ta.vec = nullptr;
    ta.out = out;
    ta.post = nullptr;
    ta.plane = L.d.plane;
    ta.nz = L.d.nz;
    ta.n = L.d.n;
    ta.deta = L.deta;
    ta.scal = guard;
    return ta;
}

// b_{l+1} = R r_l
static int mg_restrict(pcf_handle *h, int l, const float *r, const KrylovScalars *guard) {
    const MgLevel &F = h->mg->lv[l], &Cl = h->mg->lv[l + 1];
    ProfScope ps(h, PCF_PROF_MG, (2.0 + 2.0 / (Cl.cx * Cl.cy)) * 4 * (double)F.d.n);
    // 128-bit path: x aggregated in pairs (cx = 1 only arises for odd nx)
    if (Cl.cx == 2 && F.d.nx % 4 == 0 &&
        ((reinterpret_cast<uintptr_t>(r) | reinterpret_cast<uintptr_t>(F.fc)) & 15) == 0) {
        const int n4 = F.d.nx / 4;
        const dim3 blk(32, 8, 1), g((unsigned)((n4 + 31) / 32), (unsigned)((Cl.d.ny + 7) / 8), (unsigned)Cl.d.nz);
        if (Cl.cy == 2)
            k_mg_restrict4<2, 2><<<g, blk, 0, h->stream>>>(r, F.fc, F.d.nx, F.d.ny, F.d.nz, Cl.fc, Cl.b, guard);
        else
            k_mg_restrict4<2, 1><<<g, blk, 0, h->stream>>>(r, F.fc, F.d.nx, F.d.ny, F.d.nz, Cl.fc, Cl.b, guard);
        PCF_CUDA_TRY(cudaGetLastError());
        return PCF_OK;
    }
    const dim3 blk(32, 8, 1), g((unsigned)((Cl.d.nx + 31) / 32), (unsigned)((Cl.d.ny + 7) / 8), (unsigned)Cl.d.nz);
    if (Cl.cx == 2 && Cl.cy == 2)
        k_mg_restrict<float, 2, 2><<<g, blk, 0, h->stream>>>(r, F.fc, F.d.nx, F.d.ny, F.d.nz, Cl.fc, Cl.b, guard);
    else if (Cl.cx == 2)
        k_mg_restrict<float, 2, 1><<<g, blk, 0, h->stream>>>(r, F.fc, F.d.nx, F.d.ny, F.d.nz, Cl.fc, Cl.b, guard);
    else
        k_mg_restrict<float, 1, 2><<<g, blk, 0, h->stream>>>(r, F.fc, F.d.nx, F.d.ny, F.d.nz, Cl.fc, Cl.b, guard);
    PCF_CUDA_TRY(cudaGetLastError());
    return PCF_OK;
}

// s_l += P e_{l+1}
static int mg_prolong(pcf_handle *h, int l, const float *e, float *s, const KrylovScalars *guard) {
    const MgLevel &F = h->mg->lv[l], &Cl = h->mg->lv[l + 1];
    ProfScope ps(h, PCF_PROF_MG, (3.0 + 2.0 / (Cl.cx * Cl.cy)) * 4 * (double)F.d.n);
    // 128-bit path: x aggregated in pairs (cx = 1 only arises for odd nx)
    if (Cl.cx == 2 && F.d.nx % 4 == 0 &&
        ((reinterpret_cast<uintptr_t>(s) | reinterpret_cast<uintptr_t>(F.fc)) & 15) == 0) {
        const int n4 = F.d.nx / 4;
        const dim3 blk(32, 8, 1), g((unsigned)((n4 + 31) / 32), (unsigned)((F.d.ny + 7) / 8), (unsigned)F.d.nz);
        if (Cl.cy == 2)
            k_mg_prolong4<2, 2><<<g, blk, 0, h->stream>>>(e, Cl.fc, F.fc, F.d.nx, F.d.ny, F.d.nz, s, guard);
        else
            k_mg_prolong4<2, 1><<<g, blk, 0, h->stream>>>(e, Cl.fc, F.fc, F.d.nx, F.d.ny, F.d.nz, s, guard);
        PCF_CUDA_TRY(cudaGetLastError());
        return PCF_OK;
    }
    const dim3 blk(64, 4, 1), g((unsigned)((F.d.nx + 63) / 64), (unsigned)((F.d.ny + 3) / 4), (unsigned)F.d.nz);
    if (Cl.cx == 2 && Cl.cy == 2)
        k_mg_prolong<float, 2, 2><<<g, blk, 0, h->stream>>>(e, Cl.fc, F.fc, F.d.nx, F.d.ny, F.d.nz, s, guard);
    else if (Cl.cx == 2)
        k_mg_prolong<float, 2, 1><<<g, blk, 0, h->stream>>>(e, Cl.fc, F.fc, F.d.nx, F.d.ny, F.d.nz, s, guard);
    else
        k_mg_prolong<float, 1, 2><<<g, blk, 0, h->stream>>>(e, Cl.fc, F.fc, F.d.nx, F.d.ny, F.d.nz, s, guard);
    PCF_CUDA_TRY(cudaGetLastError());
    return PCF_OK;
}

// One pseudo-time step from s on level L: out = s + deta (L_h s - b), then the column solve in place.
static int mg_pseudo_step(pcf_handle *h, const MgLevel &L, const float *coef, const float *fac, const float *s,
                          float *out, const float *b, const KrylovScalars *guard, const float *post, int tag,
                          const __nv_bfloat16 *coef16 = nullptr) {
    StencilArgs<float> sa;
    sa.coef = coef;
    sa.coef16 = coef16;
    sa.tmap16 = coef16 ? L.tmap16 : nullptr;
    sa.tmap8 = coef16 ? L.tmap8 : nullptr;  // the finest level: its FP8 copy when in use
    sa.inv8 = sa.tmap8 ? h->scale8 + PCF_NCOEF : nullptr;
    sa.s = s;
    sa.out = out;
    sa.w1 = b;
    sa.deta = L.deta;
    sa.guard = guard;
    int rc = launch_stencil_dims<float, true, EPI_PSEUDO>(h, sa, L.d, tag);
    if (rc) return rc;
    ThomasArgs<float> ta = mg_targs(L, fac, out, out, guard);
    ta.post = post;
    return tag == PCF_PROF_MG ? mg_thomas<TH_T>(h, L, ta, tag) : launch_thomas<float, TH_T>(h, ta);
}

// The coarse part of the cycle from level l = m.fused_from down, as one
// cooperative launch of k_mg_coarse; *result as mg_cycle.
static int mg_coarse_launch(pcf_handle *h, int l, const KrylovScalars *guard, float **result) {
    MgState &m = *h->mg;
    CoarseArgs a{};
    a.nlev = (int)m.lv.size() - l;
    double bytes = 0;
    for (int q = 0; q < a.nlev; ++q) {
        const MgLevel &L = m.lv[l + q];
        CoarseLevel &c = a.lv[q];
        c.nx = L.d.nx;
        c.ny = L.d.ny;
        c.nz = L.d.nz;
        c.cx = L.cx;
        c.cy = L.cy;
        c.plane = L.d.plane;
        c.n = L.d.n;
        c.deta = (float)L.deta;
        c.coef = L.coef;
        c.fac = L.fac;
        c.fc = L.fc;
        c.s = L.s;
        c.t = L.t;
        c.b = L.b;
        bytes += (2.0 * 25 + 6 * 5 + 10) * 4 * (double)L.d.n;  // two stencils, two column solves, transfers
    }
    a.coarse_iters = m.coarse_iters;
    a.guard = guard;
    ProfScope ps(h, PCF_PROF_MG, bytes);
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)m.coarse_cluster);
    cfg.blockDim = dim3(kCoarseThreads);
    cfg.stream = h->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)m.coarse_cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    PCF_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_mg_coarse, a));
    h->launches += 1;
    if (a.nlev == 1)
        *result = (m.coarse_iters - 1) % 2 == 0 ? m.lv[l].s : m.lv[l].t;
    else
        *result = m.lv[l].t;
    return PCF_OK;
}

// Cycle on a coarse level l >= 1 with right-hand side lv[l].b; *result is lv[l].s or lv[l].t.
static int mg_cycle(pcf_handle *h, int l, const KrylovScalars *guard, float **result) {
    MgState &m = *h->mg;
    if (l == m.fused_from) return mg_coarse_launch(h, l, guard, result);
    const MgLevel &L = m.lv[l];
    const __nv_bfloat16 *c16 = m.bf16 ? L.coef16 : nullptr;  // level 1 only
    int rc = mg_thomas<TH_B>(h, L, mg_targs(L, L.fac, L.b, L.s, guard), PCF_PROF_MG);
    if (rc) return rc;
    if (l + 1 == (int)m.lv.size()) {
        float *cur = L.s, *oth = L.t;
        for (int q = 1; q < m.coarse_iters; ++q) {
            if ((rc = mg_pseudo_step(h, L, L.coef, L.fac, cur, oth, L.b, guard, nullptr, PCF_PROF_MG))) return rc;
            std::swap(cur, oth);
        }
        *result = cur;
        return PCF_OK;
    }
    StencilArgs<float> sa;
    sa.coef = L.coef;
    sa.coef16 = c16;
    sa.tmap16 = c16 ? L.tmap16 : nullptr;
    sa.s = L.s;
    sa.out = L.t;
    sa.w1 = L.b;
    sa.deta = 0;
    sa.guard = guard;
    if ((rc = launch_stencil_dims<float, false, EPI_RESNR>(h, sa, L.d, PCF_PROF_MG))) return rc;
    if ((rc = mg_restrict(h, l, L.t, guard))) return rc;
    float *e = nullptr;
    if ((rc = mg_cycle(h, l + 1, guard, &e))) return rc;
    if ((rc = mg_prolong(h, l, e, L.s, guard))) return rc;
    if ((rc = mg_pseudo_step(h, L, L.coef, L.fac, L.s, L.t, L.b, guard, nullptr, PCF_PROF_MG, c16))) return rc;
    *result = L.t;
    return PCF_OK;
}

// The V-cycle on the handle's grid as the right preconditioner of the FP32
// iteration: the first smoothing step forms its input by MODE (b itself, or
// the BiCGSTAB p / s update written back to bvec, as precond_apply), and the
// result (in o2) is multiplied by post (1 / fcscal) when post is set.
template <int MODE>
static int mg_precond(pcf_handle *h, const Work<float> &w, float *bvec, const KrylovScalars *guard, float **result,
                      float *o1, float *o2, const float *post) {
    MgState &m = *h->mg;
    const MgLevel &L = m.lv[0];
    const __nv_bfloat16 *c16 = m.bf16 ? h->coef16 : nullptr;
    ThomasArgs<float> ta = mg_targs(L, w.fac, bvec, o1, guard);
    ta.r = w.r;
    ta.v = w.v;
    ta.vec = bvec;
    const bool single = m.lv.size() == 1;
    if (single && m.coarse_iters <= 1) ta.post = post;
    int rc = launch_thomas<float, MODE>(h, ta);
    if (rc) return rc;
    if (single) {
        // no coarser level: the coarsest-level smoothing on this grid
        float *cur = o1, *oth = o2;
        for (int q = 1; q < m.coarse_iters; ++q) {
            if ((rc = mg_pseudo_step(h, L, w.coef, w.fac, cur, oth, bvec, guard,
                                     q + 1 == m.coarse_iters ? post : nullptr, -1, c16)))
                return rc;
            std::swap(cur, oth);
        }
        *result = cur;
        return PCF_OK;
    }
    StencilArgs<float> sa;
    sa.coef = w.coef;
    sa.coef16 = c16;
    sa.tmap16 = c16 ? L.tmap16 : nullptr;
    sa.s = o1;
    sa.out = o2;
    sa.w1 = bvec;
    sa.deta = 0;
    sa.guard = guard;
    if ((rc = launch_stencil<float, false, EPI_RESNR>(h, sa))) return rc;
    if ((rc = mg_restrict(h, 0, o2, guard))) return rc;
    float *e = nullptr;
    if ((rc = mg_cycle(h, 1, guard, &e))) return rc;
    if ((rc = mg_prolong(h, 0, e, o1, guard))) return rc;
    if ((rc = mg_pseudo_step(h, L, w.coef, w.fac, o1, o2, bvec, guard, post, -1, c16))) return rc;
    *result = o2;
    return PCF_OK;
}

static void mg_free(pcf_handle *h) {
    if (!h->mg) return;
    for (void *q : h->mg->allocs) cudaFree(q);
    h->mg->allocs.clear();
    h->mg->lv.clear();
    h->mg->maps8 = nullptr;
}

static void clear_graphs(pcf_handle *h);

// Builds (on the first call or when the level layout changes) and refreshes
// (when the operator or the smoother's step changed) the hierarchy.
// ensemble: called for a member of pcf_ensemble_solve_device (mg_fused_coarse = -1 fuses there only)
static int mg_prepare(pcf_handle *h, const pcf_params *prm, bool ensemble = false) {
    if (!(prm->mg_dtau > 0) || prm->mg_coarse_iterations < 1 || prm->mg_min_columns < 1) return PCF_EINVAL;
    if (!h->mg) h->mg = new MgState();
    MgState &m = *h->mg;
    if (m.min_columns != prm->mg_min_columns || m.lv.empty()) {
        cudaStreamSynchronize(h->stream);
        clear_graphs(h);  // captured kernels hold the old level buffers
        mg_free(h);
        MgLevel L0;
        L0.d = h->d;
        L0.dx = h->dx;
        L0.dy = h->dy;
        m.lv.push_back(L0);
        for (;;) {
            const MgLevel &F = m.lv.back();
            const int cx = (F.d.nx % 2 == 0 && F.d.nx >= 4) ? 2 : 1;
            const int cy = (F.d.ny % 2 == 0 && F.d.ny >= 4) ? 2 : 1;
            if (cx * cy == 1 || F.d.plane <= prm->mg_min_columns) break;
            MgLevel C;
            C.d.nx = F.d.nx / cx;
            C.d.ny = F.d.ny / cy;
            C.d.nz = F.d.nz;
            C.d.plane = C.d.nx * C.d.ny;
            C.d.n = (long long)C.d.plane * C.d.nz;
            C.cx = cx;
            C.cy = cy;
            C.dx = F.dx * cx;
            C.dy = F.dy * cy;
            m.lv.push_back(C);
        }
        auto alloc = [&](float **p, long long count) -> int {
            cudaError_t e = cudaMalloc((void **)p, sizeof(float) * (size_t)count);
            if (e != cudaSuccess) return pcf_set_cuda_error(e);
            m.allocs.push_back(*p);
            h->bytes += (long long)sizeof(float) * count;
            return PCF_OK;
        };
        int rc;
        if ((rc = alloc(&m.lv[0].fc, h->d.n))) return rc;
        for (size_t l = 1; l < m.lv.size(); ++l) {
            MgLevel &C = m.lv[l];
            if ((rc = alloc(&C.coef, C.d.n * PCF_NCOEF)) || (rc = alloc(&C.fac, C.d.n * 3)) ||
                (rc = alloc(&C.fc, C.d.n)) || (rc = alloc(&C.b, C.d.n)) || (rc = alloc(&C.s, C.d.n)) ||
                (rc = alloc(&C.t, C.d.n)))
                return rc;
            if (l == 1) {  // the first coarse level's BF16 copy, written by its coarsening
                float *c16 = nullptr, *maps = nullptr;
                if ((rc = alloc(&c16, (C.d.n * PCF_NCOEF + 1) / 2)) || (rc = alloc(&maps, 6 * 128 / 4))) return rc;
                C.coef16 = reinterpret_cast<__nv_bfloat16 *>(c16);
                if (make_coef16_maps(C.coef16, C.d, maps)) C.tmap16 = maps;
            }
        }
        m.min_columns = prm->mg_min_columns;
        m.version = -1;
    }
    m.coarse_iters = prm->mg_coarse_iterations;
    m.bf16 = prm->mg_operator_bf16 != 0;
    // the coarse part of the cycle in one launch: from the first level of at most
    // kCoarseColumns columns (from level 2 on when level 1 reads a BF16 copy),
    // if its columns fit the warp sweeps (nz <= 256)
    m.fused_from = -1;
    const bool fuse = prm->mg_fused_coarse > 0 || (prm->mg_fused_coarse < 0 && ensemble);
    if (fuse && h->d.nz <= 256) {
        for (int l = m.bf16 ? 2 : 1; l < (int)m.lv.size(); ++l)
            if (m.lv[l].d.plane <= kCoarseColumns) {
                if ((int)m.lv.size() - l <= kCoarseMaxLevels) m.fused_from = l;
                break;
            }
    }
    if (m.fused_from >= 0 && !m.coarse_cluster) {
        // the largest cluster the device schedules: 16 CTAs (non-portable), else 8
        PCF_CUDA_TRY(cudaFuncSetAttribute(k_mg_coarse, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        for (int size = kCoarseCluster; size >= 8 && !m.coarse_cluster; size /= 2) {
            cudaLaunchConfig_t cfg{};
            cfg.gridDim = dim3((unsigned)size);
            cfg.blockDim = dim3(kCoarseThreads);
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = (unsigned)size;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            int clusters = 0;
            if (cudaOccupancyMaxActiveClusters(&clusters, k_mg_coarse, &cfg) == cudaSuccess && clusters > 0)
                m.coarse_cluster = size;
            else
                cudaGetLastError();
        }
        if (!m.coarse_cluster) m.fused_from = -1;  // no cluster: one kernel per step
    }
    if (m.bf16 && !h->coef16) {
        // first use: allocate and convert; later assemblies and pcf_set_operator write it themselves
        const size_t bytes = sizeof(__nv_bfloat16) * (size_t)h->d.n * PCF_NCOEF;
        const cudaError_t e = cudaMalloc((void **)&h->coef16, bytes);
        if (e != cudaSuccess) {
            h->coef16 = nullptr;
            return pcf_set_cuda_error(e);
        }
        h->bytes += (long long)bytes;
        ProfScope ps(h, PCF_PROF_ASSEMBLE, 6.0 * PCF_NCOEF * (double)h->d.n);
        k_float_to_bf16<<<vec_grid(h->d.n * PCF_NCOEF), 256, 0, h->stream>>>(h->coef32, h->coef16,
                                                                              h->d.n * PCF_NCOEF);
        PCF_CUDA_TRY(cudaGetLastError());
    }
    if (m.bf16 && !m.lv[0].tmap16) {  // the finest level's maps (once per hierarchy)
        void *maps = nullptr;
        const cudaError_t e = cudaMalloc(&maps, 6 * 128);
        if (e != cudaSuccess) return pcf_set_cuda_error(e);
        m.allocs.push_back(maps);
        if (make_coef16_maps(h->coef16, h->d, maps)) m.lv[0].tmap16 = maps;
    }
    // the finest level's pseudo-time steps on an FP8 copy of its planes
    // (mg_smoother_fp8), made from the BF16 copy once per operator
    const bool fp8 = m.bf16 && prm->mg_smoother_fp8 && m.lv[0].tmap16 && h->d.nx % 16 == 0;
    if (fp8 && !h->coef8) {
        const size_t bytes = (size_t)h->d.n * PCF_NCOEF;
        cudaError_t e = cudaMalloc((void **)&h->coef8, bytes);
        if (e == cudaSuccess) e = cudaMalloc((void **)&h->scale8, 2 * PCF_NCOEF * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc((void **)&h->amax8, PCF_NCOEF * sizeof(unsigned));
        if (e != cudaSuccess) {
            cudaFree(h->coef8);
            cudaFree(h->scale8);
            h->coef8 = nullptr;
            h->scale8 = nullptr;
            return pcf_set_cuda_error(e);
        }
        h->bytes += (long long)bytes + 3 * PCF_NCOEF * 4;
        h->coef8_version = -1;
    }
    if (fp8 && !m.maps8) {  // once per hierarchy
        void *maps = nullptr;
        const cudaError_t e = cudaMalloc(&maps, 4 * 128);
        if (e != cudaSuccess) return pcf_set_cuda_error(e);
        m.allocs.push_back(maps);
        if (make_coef8_maps(h->coef8, h->d, maps)) m.maps8 = maps;
    }
    m.lv[0].tmap8 = fp8 ? m.maps8 : nullptr;
    if (m.lv[0].tmap8 && h->coef8_version != h->op_version) {
        // BF16 planes read twice (maxima, conversion), FP8 planes written
        ProfScope ps(h, PCF_PROF_ASSEMBLE, (2.0 * 2 + 1.0) * PCF_NCOEF * (double)h->d.n);
        PCF_CUDA_TRY(cudaMemsetAsync(h->amax8, 0, PCF_NCOEF * sizeof(unsigned), h->stream));
        const dim3 g((unsigned)std::max(1, num_sms() * 8 / PCF_NCOEF), PCF_NCOEF);
        k_plane_absmax<<<g, 256, 0, h->stream>>>(h->coef16, h->d.n, h->amax8);
        k_fp8_scales<<<1, 32, 0, h->stream>>>(h->amax8, h->scale8);
        k_to_fp8<<<g, 256, 0, h->stream>>>(h->coef16, h->d.n, h->scale8, h->coef8);
        h->launches += 3;
        PCF_CUDA_TRY(cudaGetLastError());
        h->coef8_version = h->op_version;
    }
    for (MgLevel &L : m.lv) L.deta = prm->mg_dtau / (2 * (1 / (L.dx * L.dx) + 1 / (L.dy * L.dy)));
    // the finest level's pivots are the handle's (shared with the reference preconditioner)
    int rc = ensure_factors(h, m.lv[0].deta);
    if (rc) return rc;
    if (m.version == h->op_version && m.dtau == prm->mg_dtau) return PCF_OK;
    // finest level: fcscal in FP32
    {
        ProfScope ps(h, PCF_PROF_ASSEMBLE, 12.0 * (double)h->d.n);
        k_to_float<<<vec_grid(h->d.n), 256, 0, h->stream>>>(h->fc64, m.lv[0].fc, h->d.n, 1.0);
        PCF_CUDA_TRY(cudaGetLastError());
    }
    for (size_t l = 1; l < m.lv.size(); ++l) {
        const MgLevel &F = m.lv[l - 1];
        MgLevel &C = m.lv[l];
        ProfScope ps(h, PCF_PROF_ASSEMBLE, (26.0 * (l == 1 ? 8 : 4) + 32.0 / (C.cx * C.cy)) * (double)F.d.n);
        const unsigned gf = vec_grid(C.d.n);
        const dim3 gc((unsigned)((C.d.n + 127) / 128), 5, 1);  // x: coarse cells, y: the five dz groups
#define PCF_MG_BUILD(CX, CY)                                                                                          \
    do {                                                                                                              \
        k_mg_fc<float, CX, CY><<<gf, 256, 0, h->stream>>>(F.fc, F.d.nx, F.d.ny, F.d.nz, C.fc);                        \
        if (l == 1)                                                                                                   \
            k_mg_coarsen<double, CX, CY><<<gc, 128, 0, h->stream>>>(h->coef64, h->fc64, F.d.nx, F.d.ny, F.d.nz, C.fc, \
                                                                    C.coef, C.coef16);                                \
        else                                                                                                          \
            k_mg_coarsen<float, CX, CY><<<gc, 128, 0, h->stream>>>(F.coef, F.fc, F.d.nx, F.d.ny, F.d.nz, C.fc,       \
                                                                   C.coef, nullptr);                                  \
    } while (0)
        if (C.cx == 2 && C.cy == 2)
            PCF_MG_BUILD(2, 2);
        else if (C.cx == 2)
            PCF_MG_BUILD(2, 1);
        else
            PCF_MG_BUILD(1, 2);
#undef PCF_MG_BUILD
        PCF_CUDA_TRY(cudaGetLastError());
        k_mg_factors<<<(C.d.plane + 127) / 128, 128, 0, h->stream>>>(C.d.plane, C.d.nz, C.d.n, C.deta, C.coef, C.fac);
        PCF_CUDA_TRY(cudaGetLastError());
        h->launches += 2;
    }
    m.version = h->op_version;
    m.dtau = prm->mg_dtau;
    return PCF_OK;
}

// Tunes the stencil families that a solve with these settings launches
// (before its iteration batches are captured).
static int autotune_handle(pcf_handle *h, const pcf_params *prm) {
    int rc;
    if (prm->precision == PCF_PRECISION_MIXED) {
        if ((rc = tune_stencil<float, false, true>(h, h->d, h->coefB32, h->za32, h->zb32, h->s32))) return rc;
        if (prm->preconditioner && !prm->multigrid &&
            (rc = tune_stencil<float, true, false>(h, h->d, h->coef32, h->za32, h->zb32, h->s32)))
            return rc;
        if (prm->multigrid && h->mg) {
            if ((rc = tune_stencil<float, true, false>(h, h->d, h->coef32, h->za32, h->zb32, h->s32))) return rc;
            if ((rc = tune_stencil<float, false, false>(h, h->d, h->coef32, h->za32, h->zb32, h->s32))) return rc;
            for (size_t l = 1; l < h->mg->lv.size(); ++l) {
                const MgLevel &L = h->mg->lv[l];
                if ((rc = tune_stencil<float, false, false>(h, L.d, L.coef, L.s, L.t, L.b))) return rc;
                if ((rc = tune_stencil<float, true, false>(h, L.d, L.coef, L.s, L.t, L.b))) return rc;
            }
        }
    } else if (prm->preconditioner) {
        if ((rc = tune_stencil<double, true, false>(h, h->d, h->coef64, h->za64, h->zb64, h->s64))) return rc;
    }
    // FP64 applies: the reference loop and the true residual of the mixed solve
    return tune_stencil<double, false, false>(h, h->d, h->coef64, h->za64, h->zb64, h->s64);
}

struct LoopCfg {
    int precond, pc_iters;
    double deta;
    int flex;      // accumulate x from the preconditioned directions (FP32 inner loop)
    int reliable;  // fold into the FP64 solution and restart r from the true residual
    int mg = 0;    // multigrid V-cycle as the preconditioner (FP32 loop only)
    int learned_pc = 0;  // learned stage after the preconditioner (FP32 loop only)
};

// The learned preconditioner stage on the preconditioner's s-space output z
// (in place): r2 = bvec - A z, c = N(r2), z = (z + c) / fcscal.  The network
// is bias-free, hence N(a r2) = a N(r2), and needs no normalisation of r2.
static int learned_stage(pcf_handle *h, const Work<float> &w, const float *bvec, float *z, const KrylovScalars *guard) {
    float *r2 = h->lr32, *cc = h->lr32 + h->d.n;
    StencilArgs<float> sa;
    sa.coef = w.coef;
    sa.s = z;
    sa.out = r2;
    sa.w1 = bvec;
    sa.deta = 0;
    sa.guard = guard;
    int rc = launch_stencil<float, false, EPI_RESNR>(h, sa);
    if (rc) return rc;
    {
        ProfScope ps(h, PCF_PROF_LEARNED, 8.0 * h->d.n);
        h->launches += 6;  // gather, 3 GEMMs, 2 convolutions (the scope counts the scatter)
        if ((rc = pcf_net_apply_device(h->net, r2, h->d.nx, h->d.ny, h->d.nz, 1.0, 1.0, 0.0, cc, 0, h->stream)))
            return rc;
    }
    h->launches += 1;
    k_learned_combine<<<vec_grid(h->d.n), 256, 0, h->stream>>>(z, cc, w.post, h->d.n, guard);
    PCF_CUDA_TRY(cudaGetLastError());
    return PCF_OK;
}

// Profiler bytes of the FP64 true-residual applies of `nupdates` reliable
// updates: 25 coefficient planes + x + b + r words per cell.
static void reliable_bytes(pcf_handle *h, int nupdates) {
    if (h->prof_on && h->prof && nupdates > 0)
        h->prof_acc[PCF_PROF_RELIABLE].bytes += (double)nupdates * 28.0 * sizeof(double) * (double)h->d.n;
}

// Reliable update (mixed precision): x64 += bnorm64 x32, r64 = b - A64 x64
// with the FP64 convergence test, r32 = r64 / bnorm64, <r32, r0>.  The three
// launches return at once unless the last FIN_RESID raised the update flag.
static int reliable_update(pcf_handle *h) {
    KrylovScalars *sc = h->scal32;
    h->launches += 1;
    k_ru_fold<<<vec_grid(h->d.n), 256, 0, h->stream>>>(h->x32, h->x64, h->fc64, h->d.n, sc);
    PCF_CUDA_TRY(cudaGetLastError());
    StencilArgs<double> a;
    a.coef = h->coef64;
    a.s = h->x64;
    a.out = h->w64;
    a.w1 = h->b64;
    a.deta = 0;
    a.guard = sc;
    a.guard_update = 1;
    a.red = red(h, sc, FIN_RU_TRUE);
    int rc = launch_stencil<double, false, EPI_RESID>(h, a);
    if (rc) return rc;
    h->launches += 1;
    k_ru_convert<<<vec_grid(h->d.n), 256, 0, h->stream>>>(h->w64, h->r32, h->r032, h->d.n, red(h, sc, FIN_RU_RHO));
    PCF_CUDA_TRY(cudaGetLastError());
    return PCF_OK;
}

// One BiCGSTAB iteration, apply_bicgstab!.jl:81-143.
template <typename T>
static int bicgstab_iteration(pcf_handle *h, const Work<T> &w, const LoopCfg &c) {
    int rc;
    T *z = nullptr, *zp = nullptr;
    // p = r + beta (p - omega v); z = M p
    if (c.precond) {
        if constexpr (sizeof(T) == 4) {
            const float *post = c.learned_pc ? nullptr : w.post;
            if (c.mg)
                rc = mg_precond<TH_PUPD>(h, w, w.p, w.scal, &z, w.za, w.zb, post);
            else
                rc = precond_apply<T, TH_PUPD>(h, w, w.p, c.pc_iters, c.deta, w.scal, &z, nullptr, nullptr, post);
            if (!rc && c.learned_pc) rc = learned_stage(h, w, w.p, z, w.scal);
        } else {
            rc = precond_apply<T, TH_PUPD>(h, w, w.p, c.pc_iters, c.deta, w.scal, &z, nullptr, nullptr, w.post);
        }
        zp = z;
    } else {
        h->launches += 1;
        k_axpy_noprec<T, TH_PUPD><<<vec_grid(h->d.n), 256, 0, h->stream>>>(w.r, w.v, w.p, h->d.n, w.scal);
        rc = cudaGetLastError() == cudaSuccess ? PCF_OK : PCF_ECUDA;
        z = w.p;
        zp = z;
    }
    if (rc) return rc;
    // v = A z; alpha = <r, r0> / <v, r0>
    {
        StencilArgs<T> sa;
        sa.coef = w.coefT;
        sa.s = z;
        sa.out = w.v;
        sa.w1 = w.r0;
        sa.deta = 0;
        sa.red = red(h, w.scal, FIN_ALPHA);
        sa.guard = w.scal;
        rc = apply_total<T, EPI_DOT1>(h, sa, w.post != nullptr);
        if (rc) return rc;
    }
    // s = r - alpha v; z = M s
    if (c.precond) {
        bool done = false;
        const T *post = w.post;
        if constexpr (sizeof(T) == 4) {
            if (c.learned_pc) post = nullptr;
            if (c.mg) {
                rc = mg_precond<TH_SUPD>(h, w, w.s, w.scal, &z, w.zc, w.zd, post);
                done = true;
            }
        }
        if (!done)
            rc = precond_apply<T, TH_SUPD>(h, w, w.s, c.pc_iters, c.deta, w.scal, &z, c.flex ? w.zc : w.za,
                                           c.flex ? w.zd : w.zb, post);
        if constexpr (sizeof(T) == 4) {
            if (!rc && c.learned_pc) rc = learned_stage(h, w, w.s, z, w.scal);
        }
    } else {
        h->launches += 1;
        k_axpy_noprec<T, TH_SUPD><<<vec_grid(h->d.n), 256, 0, h->stream>>>(w.r, w.v, w.s, h->d.n, w.scal);
        rc = cudaGetLastError() == cudaSuccess ? PCF_OK : PCF_ECUDA;
        z = w.s;
    }
    if (rc) return rc;
    // t = A z; omega = <t, s> / <t, t>
    {
        StencilArgs<T> sa;
        sa.coef = w.coefT;
        sa.s = z;
        sa.out = w.t;
        sa.w1 = w.s;
        sa.deta = 0;
        sa.red = red(h, w.scal, FIN_OMEGA);
        sa.guard = w.scal;
        rc = apply_total<T, EPI_DOT2>(h, sa, w.post != nullptr);
        if (rc) return rc;
    }
    // x += alpha p + omega s; r = s - omega t; residual test, beta
    {
        UpdateArgs<T> ua;
        ua.x = w.x;
        ua.r = w.r;
        ua.p = w.p;
        ua.s = w.s;
        ua.t = w.t;
        ua.r0 = w.r0;
        ua.zp = zp;
        ua.zs = z;
        ua.n = h->d.n;
        ua.red = red(h, w.scal, FIN_RESID);
        ua.scal = w.scal;
        ProfScope ps(h, sizeof(T) == 4 ? PCF_PROF_UPDATE32 : PCF_PROF_UPDATE64, 7.0 * sizeof(T) * (double)h->d.n);
        constexpr int VU = sizeof(T) == 4 ? 4 : 2;
        const bool vec = h->d.n % VU == 0;
        const long long units = vec ? h->d.n / VU : h->d.n;
        const unsigned grid = (unsigned)std::max<long long>(1, std::min<long long>((units + 255) / 256, 16LL * num_sms()));
        if (c.flex) {
            if (vec) k_update<T, true, VU><<<grid, 256, 0, h->stream>>>(ua);
            else k_update<T, true, 1><<<grid, 256, 0, h->stream>>>(ua);
        } else {
            if (vec) k_update<T, false, VU><<<grid, 256, 0, h->stream>>>(ua);
            else k_update<T, false, 1><<<grid, 256, 0, h->stream>>>(ua);
        }
        PCF_CUDA_TRY(cudaGetLastError());
    }
    if (c.reliable) return reliable_update(h);
    return PCF_OK;
}

struct RunOut {
    int iters, converged, status, nupdates;
    double res, b_norm;
};

// A batch of BiCGSTAB iterations captured as a CUDA graph.  The kernels'
// arguments are the handle's fixed buffers and the loop configuration, so one
// graph per configuration serves every later solve on the handle.
struct GraphKey {
    int tsize, precond, pc_iters, flex, reliable, pi, batch;
    double deta;
    int mg, mg_levels, mg_coarse_iters, mg_bf16;
    const void *net;  // the learned stage's network (null: no stage)
    bool operator==(const GraphKey &o) const {
        return tsize == o.tsize && precond == o.precond && pc_iters == o.pc_iters && flex == o.flex &&
               reliable == o.reliable && pi == o.pi && batch == o.batch && deta == o.deta && mg == o.mg &&
               mg_levels == o.mg_levels && mg_coarse_iters == o.mg_coarse_iters && mg_bf16 == o.mg_bf16 &&
               net == o.net;
    }
};
struct GraphEntry {
    GraphKey key;
    cudaGraphExec_t exec;
    long long launches;
};
struct GraphCache {
    std::vector<GraphEntry> entries;
};

template <typename T>
static int batch_graph(pcf_handle *h, const Work<T> &w, const LoopCfg &c, const GraphKey &key,
                       cudaGraphExec_t *out) {
    if (!h->gcache) h->gcache = new GraphCache();
    for (const GraphEntry &e : h->gcache->entries)
        if (e.key == key) {
            *out = e.exec;
            h->graph_launches = e.launches;
            return PCF_OK;
        }
    const long long l0 = h->launches;
    PCF_CUDA_TRY(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int rc = PCF_OK;
    for (int q = 0; q < key.batch && rc == PCF_OK; ++q) rc = bicgstab_iteration<T>(h, w, c);
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(h->stream, &graph);
    const long long nlaunch = h->launches - l0;
    h->launches = l0;  // captured, not launched
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (ec != cudaSuccess) return pcf_set_cuda_error(ec);
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) return pcf_set_cuda_error(ei);
    h->gcache->entries.push_back({key, exec, nlaunch});
    h->graph_launches = nlaunch;
    *out = exec;
    return PCF_OK;
}

static void clear_graphs(pcf_handle *h) {
    if (!h->gcache) return;
    for (const GraphEntry &e : h->gcache->entries) cudaGraphExecDestroy(e.exec);
    h->gcache->entries.clear();
}

// A complete BiCGSTAB run on A x = b (b in w.r on entry is not required: b
// is the `b` argument), x0 = 0.  On convergence x <- M x as at
// apply_bicgstab!.jl:132-135.  Result vector: *xout (x or a z buffer).
// The part of a run before its iterations: the scalar block and
// r0 = r = p = b, x = 0 (apply_bicgstab!.jl:44-67).
template <typename T>
static int run_start(pcf_handle *h, const Work<T> &w, const T *b, double tol, int maxit, const LoopCfg &c,
                     int hist_off, double hist_scale, double bnorm64, double ru_delta, int restart_every) {
    KrylovScalars init;
    std::memset(&init, 0, sizeof(init));
    init.tol = tol;
    init.maxit = maxit;
    init.ncell = (double)h->d.n;
    init.hist = h->hist;
    init.hist_cap = kHistCap;
    init.hist_off = hist_off;
    init.hist_scale = hist_scale;
    init.reliable = c.reliable;
    init.bnorm64 = bnorm64;
    init.ru_delta = ru_delta;
    init.restart_every = restart_every;
    PCF_CUDA_TRY(cudaMemcpyAsync(w.scal, &init, sizeof(init), cudaMemcpyHostToDevice, h->stream));
    PCF_CUDA_TRY(cudaMemsetAsync(w.v, 0, sizeof(T) * h->d.n, h->stream));
    h->launches += 1;
    k_init<T><<<vec_grid(h->d.n), 256, 0, h->stream>>>(b, w.x, w.r, w.r0, w.p, h->d.n, red(h, w.scal, FIN_INIT));
    PCF_CUDA_TRY(cudaGetLastError());
    return PCF_OK;
}

// The part of a run after its iterations (the stream is drained here): the
// outcome, the residual history and, for the reference form, x <- M x
// (apply_bicgstab!.jl:132-135).
template <typename T>
static int run_finish(pcf_handle *h, const Work<T> &w, const LoopCfg &c, bool precondition_unconverged,
                      int hist_off, T **xout, RunOut *out) {
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    // the latest status (a batch issued after convergence leaves it unchanged)
    PCF_CUDA_TRY(cudaMemcpy(h->h_scal, w.scal, sizeof(KrylovScalars), cudaMemcpyDeviceToHost));
    const KrylovScalars s = *h->h_scal;
    if (s.status == PCF_ECUDA) {
        // a stencil block that gave up on its copies left before the reduction,
        // so the reduction ticket was not returned to zero
        PCF_CUDA_TRY(cudaMemsetAsync(h->ticket, 0, sizeof(unsigned int) * 4, h->stream));
    }
    h->prof_iter = -1;
    prof_flush(h, s.iter);
    h->hist_len = std::min(hist_off + s.iter, kHistCap);
    out->iters = s.iter;
    out->converged = s.converged;
    out->status = s.status;
    out->res = c.reliable ? s.res_true : (s.b_norm > 0 ? s.res / s.b_norm : 0.0);
    out->b_norm = s.b_norm;
    out->nupdates = s.nupdates;
    *xout = w.x;
    const bool finish = s.converged || (precondition_unconverged && s.status == PCF_OK);
    if (finish && s.iter > 0 && c.precond && !c.flex) {
        T *z = nullptr;
        int rc = precond_apply<T, TH_B>(h, w, w.x, c.pc_iters, c.deta, nullptr, &z);
        if (rc) return rc;
        *xout = z;
    }
    return PCF_OK;
}

static GraphKey graph_key(const pcf_handle *h, int tsize, const LoopCfg &c, bool pi, int check_interval) {
    return GraphKey{tsize, c.precond, c.pc_iters, c.flex, c.reliable, pi, check_interval, c.deta, c.mg,
                    c.mg && h->mg ? (int)h->mg->lv.size() : 0, c.mg && h->mg ? h->mg->coarse_iters : 0,
                    c.mg && h->mg ? (int)h->mg->bf16 | (h->mg->lv[0].tmap8 ? 2 : 0) | (h->mg->fused_from + 1) << 2 : 0,
                    c.learned_pc ? (const void *)h->net : nullptr};
}

// A complete BiCGSTAB run: run_start, the iteration batches, run_finish.
template <typename T>
static int bicgstab_run(pcf_handle *h, const Work<T> &w, const T *b, double tol, int maxit, const LoopCfg &c,
                        int check_interval, bool precondition_unconverged, T **xout, RunOut *out,
                        int hist_off = 0, double hist_scale = 1.0, double bnorm64 = 0.0, double ru_delta = 0.0,
                        int restart_every = 0) {
    int rc0 = run_start<T>(h, w, b, tol, maxit, c, hist_off, hist_scale, bnorm64, ru_delta, restart_every);
    if (rc0) return rc0;
    if (check_interval < 1) check_interval = 16;
    // Iterations are issued in batches of check_interval; a batch is a CUDA
    // graph (captured once per handle and loop configuration) unless per-launch
    // profiling is on.  The status word of batch b is read back while batch
    // b + 1 is already queued, so the GPU never drains between batches; the
    // batch queued after convergence returns at once.
    const GraphKey key = graph_key(h, (int)sizeof(T), c, w.post != nullptr, check_interval);
    cudaGraphExec_t gexec = nullptr;
    if (!h->prof_on) {
        int rc = batch_graph<T>(h, w, c, key, &gexec);
        if (rc) return rc;
    }
    int launched = 0, inflight = 0, slot = 0;
    int done_seen = 0;
    KrylovScalars last;
    std::memset(&last, 0, sizeof(last));
    while (!done_seen) {
        if (launched < maxit) {
            const int nb = std::min(check_interval, maxit - launched);
            if (gexec && nb == check_interval) {
                h->launches += h->graph_launches;
                PCF_CUDA_TRY(cudaGraphLaunch(gexec, h->stream));
            } else {
                for (int q = 0; q < nb; ++q) {
                    h->prof_iter = launched + q;
                    int rc = bicgstab_iteration<T>(h, w, c);
                    if (rc) return rc;
                }
            }
            launched += nb;
            PCF_CUDA_TRY(cudaMemcpyAsync(h->h_scal + slot, w.scal, sizeof(KrylovScalars), cudaMemcpyDeviceToHost,
                                         h->stream));
            PCF_CUDA_TRY(cudaEventRecord(h->ev[5 + slot], h->stream));
            slot ^= 1;
            inflight += 1;
        }
        if (inflight == 0) break;
        // wait for the older of the (at most two) batches in flight
        if (inflight == 2 || launched >= maxit) {
            const int old = (inflight == 2) ? slot : slot ^ 1;
            PCF_CUDA_TRY(cudaEventSynchronize(h->ev[5 + old]));
            last = h->h_scal[old];
            inflight -= 1;
            if (last.done) done_seen = 1;
            if (launched >= maxit && inflight == 0) break;
        }
    }
    return run_finish<T>(h, w, c, precondition_unconverged, hist_off, xout, out);
}

// ------------------------------------------------------- small kernels --

__global__ void k_to_float(const double *__restrict__ a, float *__restrict__ b, long long n, double scale) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = (float)(a[i] * scale);
}
__global__ void k_to_double(const float *__restrict__ a, double *__restrict__ b, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = (double)a[i];
}
// x += scale * fc * e (fc may be null: 1)
__global__ void k_axpy_f2d(const float *__restrict__ e, double *__restrict__ x, const double *__restrict__ fc,
                           long long n, double scale) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] += (double)e[i] * scale * (fc ? fc[i] : 1.0);
}
// pi = s / fcscal in FP32 (for the difference-form operator entry point)
__global__ void k_to_pi(const double *__restrict__ s, const float *__restrict__ rfc, float *__restrict__ pi,
                        long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        pi[i] = (float)(s[i] * (double)rfc[i]);
}
__global__ void k_coef_to_float(const double *__restrict__ a, float *__restrict__ b, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}
// dpip = (1/dt) * s / sqrt(pbar^2 / rhobar) on the interior (solve_poisson!.jl:65-72);
// dst is haloed with offsets (ox, oy, oz) and pitches (sx, sy), or compact.
__global__ void k_unscale(const double *__restrict__ x, const double *__restrict__ pbar,
                          const double *__restrict__ rhobar, double dtinv, int nx, int ny, int nz, int nbx, int nby,
                          int nbz, int nxx, int nyy, double *__restrict__ dst, int ox, int oy, int oz, int sx, int sy) {
    const long long n = (long long)nx * ny * nz;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const unsigned cu = (unsigned)c, ux = (unsigned)nx, uy = (unsigned)ny;  // n < 2^31 (see k_build_diff)
        const int i = (int)(cu % ux), j = (int)((cu / ux) % uy), k = (int)(cu / (ux * uy));
        const long long hh = (i + nbx) + (long long)nxx * ((j + nby) + (long long)nyy * (k + nbz));
        const double pb = pbar[hh];
        const double sol = x[c] / sqrt(pb * pb / rhobar[hh]);
        dst[(i + ox) + (long long)sx * ((j + oy) + (long long)sy * (k + oz))] = dtinv * sol;
    }
}

}  // namespace pcf

using namespace pcf;

// ================================================================== C ABI ==

extern "C" {

const char *pcf_strerror(int code) {
    switch (code) {
        case PCF_OK: return "success";
        case PCF_EINVAL: return "invalid argument";
        case PCF_ENOMEM: return "device memory allocation failed";
        case PCF_ECUDA: return "CUDA runtime error";
        case PCF_ENOTREADY: return "grid or background not set";
        case PCF_EBREAKDOWN: return "BiCGSTAB breakdown (zero or non-finite scalar)";
        case PCF_ENONFINITE: return "non-finite value in the inputs or the residual";
        case PCF_ENODEVICE: return "no usable sm_100 CUDA device";
        case PCF_ERANGE: return "size beyond a documented limit";
        default: return "unknown error";
    }
}

int pcf_params_default(pcf_params *p) {
    if (!p) return PCF_EINVAL;
    // PoissonNamelist.jl:48-56
    p->tolerance = 1.0e-8;
    p->poisson_iterations = 1000;
    p->preconditioner = 1;
    p->dtau = 1.0;
    p->preconditioner_iterations = 2;
    p->tolerance_is_relative = 0;
    p->damp_horizontal_wind_on_rhs = 0;  // SpongeNamelist default
    p->precision = PCF_PRECISION_FP64;
    p->residual = PCF_RESIDUAL_RECURSIVE;
    p->inner_tolerance = 1.0e-2;
    p->max_refinements = 5;
    p->learned = 0;
    p->check_interval = 4;
    p->restart_interval = 1;
    p->multigrid = 0;
    p->mg_dtau = 2.5;
    p->mg_coarse_iterations = 4;
    p->mg_min_columns = 16;
    p->autotune = 0;
    p->mg_operator_bf16 = 1;
    p->mg_fused_coarse = -1;
    p->mg_smoother_fp8 = 0;
    return PCF_OK;
}

static int dalloc(pcf_handle *h, void **p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) return pcf_set_cuda_error(e);
    h->bytes += (long long)bytes;
    return PCF_OK;
}

int pcf_destroy(pcf_handle *h) {
    if (!h) return PCF_OK;
    int dev = h->dims.device;
    cudaSetDevice(dev);
    void *ptrs[] = {h->jac, h->met13, h->met23, h->met33, h->pbar, h->rhobar, h->thetabar, h->n2, h->rho, h->betar,
                    h->p, h->coef64, h->coef32, h->fac64, h->fac32, h->coefB32, h->fc64, h->rfc32, h->fch, h->rfch, h->stage, h->corr, h->istage, h->coef16, h->coef8, h->scale8, h->amax8, h->lr32,
                    h->x64, h->r64, h->r064, h->p64, h->v64, h->s64,
                    h->t64, h->za64, h->zb64, h->b64, h->w64, h->x32, h->r32, h->r032, h->p32, h->v32, h->s32,
                    h->t32, h->za32, h->zb32, h->zc32, h->zd32, h->partials, h->ticket, h->scal64, h->scal32,
                    h->dot_out,
                    h->hist};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    if (h->h_scal) cudaFreeHost(h->h_scal);
    if (h->gcache) {
        for (const GraphEntry &e : h->gcache->entries) cudaGraphExecDestroy(e.exec);
        delete h->gcache;
    }
    if (h->mg) {
        mg_free(h);
        delete h->mg;
    }
    if (h->prof) {
        for (cudaEvent_t e : h->prof->pool) cudaEventDestroy(e);
        delete h->prof;
    }
    for (auto &e : h->ev)
        if (e) cudaEventDestroy(e);
    for (auto &e : h->slab_ev)
        if (e) cudaEventDestroy(e);
    if (h->stream) cudaStreamDestroy(h->stream);
    if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
    delete h;
    return PCF_OK;
}

int pcf_create(pcf_handle **out, const pcf_dims *dims) {
    if (!out || !dims) return PCF_EINVAL;
    *out = nullptr;
    // nz >= 4: the four vertical boundary cases of the operator must be distinct levels.
    if (dims->nx < 1 || dims->ny < 1 || dims->nz < 4 || dims->nbx < 1 || dims->nby < 1 || dims->nbz < 2)
        return PCF_EINVAL;
    if (dims->model < 0 || dims->model > 2) return PCF_EINVAL;
    // cell indices are decomposed in 32 bits (an FP64 operator of 2^31 cells
    // would need 430 GB, beyond any single GPU's memory anyway)
    const long long haloed = (long long)(dims->nx + 2 * dims->nbx) * (dims->ny + 2 * dims->nby) *
                             (long long)(dims->nz + 2 * dims->nbz);
    if (haloed >= (1LL << 31)) return PCF_ERANGE;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || dims->device < 0 || dims->device >= ndev) return PCF_ENODEVICE;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dims->device) != cudaSuccess || prop.major < 10) return PCF_ENODEVICE;
    PCF_CUDA_TRY(cudaSetDevice(dims->device));
    // the staged V-cycle stencils' shared-memory limit, set here rather than
    // at a first launch that may fall inside a graph capture
    stencil_bulk_ready<float, 4, 32, 4, false, EPI_RESNR, false>();
    stencil_bulk_ready<float, 4, 32, 4, true, EPI_PSEUDO, false>();
    stencil_bulk_ready<float, 2, 32, 4, false, EPI_RESNR, false>();
    stencil_bulk_ready<float, 2, 32, 4, true, EPI_PSEUDO, false>();
    stencil_bulk_ready<float, 4, 32, 4, true, EPI_PSEUDO, false, 3>();
    stencil_bulk_ready<float, 2, 32, 4, true, EPI_PSEUDO, false, 3>();

    pcf_handle *h = new pcf_handle;
    std::memset(h, 0, sizeof(*h));
    h->coef8_version = -1;
    h->dims = *dims;
    h->d.nx = dims->nx;
    h->d.ny = dims->ny;
    h->d.nz = dims->nz;
    h->d.n = (long long)dims->nx * dims->ny * dims->nz;
    h->d.plane = dims->nx * dims->ny;
    h->nxx = dims->nx + 2 * dims->nbx;
    h->nyy = dims->ny + 2 * dims->nby;
    h->nzz = dims->nz + 2 * dims->nbz;
    h->nh = (long long)h->nxx * h->nyy * h->nzz;
    h->fac_deta = std::nan("");
    h->prof_iter = -1;
    h->prof = new ProfState();
    int rc = PCF_OK;
    auto fail = [&](int code) {
        pcf_destroy(h);
        return code;
    };
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(PCF_ECUDA);
    if (cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking) != cudaSuccess) return fail(PCF_ECUDA);
    for (auto &e : h->ev)
        if (cudaEventCreate(&e) != cudaSuccess) return fail(PCF_ECUDA);
    for (auto &e : h->slab_ev)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return fail(PCF_ECUDA);
    const size_t nh8 = sizeof(double) * (size_t)h->nh;
    const size_t n8 = sizeof(double) * (size_t)h->d.n, n4 = sizeof(float) * (size_t)h->d.n;
    double **fields[] = {&h->jac, &h->met13, &h->met23, &h->met33, &h->pbar, &h->rhobar, &h->thetabar, &h->n2,
                         &h->rho, &h->betar, &h->p};
    for (double **f : fields)
        if ((rc = dalloc(h, (void **)f, nh8))) return fail(rc);
    if ((rc = dalloc(h, (void **)&h->coef64, n8 * PCF_NCOEF))) return fail(rc);
    if ((rc = dalloc(h, (void **)&h->coef32, n4 * PCF_NCOEF))) return fail(rc);
    if ((rc = dalloc(h, (void **)&h->fac64, n8 * 3))) return fail(rc);
    if ((rc = dalloc(h, (void **)&h->fac32, n4 * 3))) return fail(rc);
    if ((rc = dalloc(h, (void **)&h->coefB32, n4 * PCF_NCOEF))) return fail(rc);
    if ((rc = dalloc(h, (void **)&h->fc64, n8))) return fail(rc);
    if ((rc = dalloc(h, (void **)&h->rfc32, n4))) return fail(rc);
    if ((rc = dalloc(h, (void **)&h->fch, nh8))) return fail(rc);
    if ((rc = dalloc(h, (void **)&h->rfch, nh8))) return fail(rc);
    double **v64[] = {&h->x64, &h->r64, &h->r064, &h->p64, &h->v64, &h->s64, &h->t64, &h->za64, &h->zb64, &h->b64,
                      &h->w64};
    for (double **v : v64)
        if ((rc = dalloc(h, (void **)v, n8))) return fail(rc);
    float **v32[] = {&h->x32, &h->r32, &h->r032, &h->p32, &h->v32, &h->s32, &h->t32, &h->za32, &h->zb32,
                     &h->zc32, &h->zd32};
    for (float **v : v32)
        if ((rc = dalloc(h, (void **)v, n4))) return fail(rc);
    if ((rc = dalloc(h, (void **)&h->partials, sizeof(double) * 2 * kMaxPartials))) return fail(rc);
    if ((rc = dalloc(h, (void **)&h->ticket, sizeof(unsigned int) * 4))) return fail(rc);
    if ((rc = dalloc(h, (void **)&h->scal64, sizeof(KrylovScalars)))) return fail(rc);
    if ((rc = dalloc(h, (void **)&h->scal32, sizeof(KrylovScalars)))) return fail(rc);
    if ((rc = dalloc(h, (void **)&h->dot_out, sizeof(double) * 4))) return fail(rc);
    if ((rc = dalloc(h, (void **)&h->hist, sizeof(double) * kHistCap))) return fail(rc);
    if (cudaMallocHost((void **)&h->h_scal, 2 * sizeof(KrylovScalars)) != cudaSuccess) return fail(PCF_ENOMEM);
    if (cudaMemsetAsync(h->ticket, 0, sizeof(unsigned int) * 4, h->stream) != cudaSuccess) return fail(PCF_ECUDA);
    // fields a caller may legitimately leave unset read as zero
    if (cudaMemsetAsync(h->thetabar, 0, nh8, h->stream) != cudaSuccess) return fail(PCF_ECUDA);
    if (cudaMemsetAsync(h->p, 0, nh8, h->stream) != cudaSuccess) return fail(PCF_ECUDA);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return fail(PCF_ECUDA);
    *out = h;
    return PCF_OK;
}

long long pcf_device_bytes(const pcf_handle *h) { return h ? h->bytes : 0; }

int pcf_set_grid(pcf_handle *h, double dx, double dy, double dz, const double *jac, const double *met13,
                 const double *met23, const double *met33) {
    if (!h || !jac || !met13 || !met23 || !met33 || !(dx > 0) || !(dy > 0) || !(dz > 0)) return PCF_EINVAL;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    const size_t b = sizeof(double) * (size_t)h->nh;
    h->dx = dx;
    h->dy = dy;
    h->dz = dz;
    PCF_CUDA_TRY(cudaMemcpyAsync(h->jac, jac, b, cudaMemcpyHostToDevice, h->stream));
    PCF_CUDA_TRY(cudaMemcpyAsync(h->met13, met13, b, cudaMemcpyHostToDevice, h->stream));
    PCF_CUDA_TRY(cudaMemcpyAsync(h->met23, met23, b, cudaMemcpyHostToDevice, h->stream));
    PCF_CUDA_TRY(cudaMemcpyAsync(h->met33, met33, b, cudaMemcpyHostToDevice, h->stream));
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->grid_set = 1;
    h->fac_deta = std::nan("");
    return PCF_OK;
}

int pcf_set_background(pcf_handle *h, const double *pbar, const double *rhobar, const double *thetabar,
                       const double *n2) {
    if (!h || !pbar || !rhobar || !n2) return PCF_EINVAL;
    if (h->dims.model == PCF_MODEL_COMPRESSIBLE && !thetabar) return PCF_EINVAL;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    const size_t b = sizeof(double) * (size_t)h->nh;
    PCF_CUDA_TRY(cudaMemcpyAsync(h->pbar, pbar, b, cudaMemcpyHostToDevice, h->stream));
    PCF_CUDA_TRY(cudaMemcpyAsync(h->rhobar, rhobar, b, cudaMemcpyHostToDevice, h->stream));
    PCF_CUDA_TRY(cudaMemcpyAsync(h->n2, n2, b, cudaMemcpyHostToDevice, h->stream));
    if (thetabar) PCF_CUDA_TRY(cudaMemcpyAsync(h->thetabar, thetabar, b, cudaMemcpyHostToDevice, h->stream));
    int rc = fcscal_halo(h, 1);
    if (rc) return rc;
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->background_set = 1;
    return PCF_OK;
}

// Assembles z-chunks [c0, c1) (c1 < 0: to the top); the operator is set
// once the last chunk is queued.
static int assemble_chunks(pcf_handle *h, double dt, double rf, int damp_h, int c0, int c1) {
    const int nchunks = (h->d.nz + pcf_assemble_chunk_levels() - 1) / pcf_assemble_chunk_levels();
    if (c1 < 0 || c1 > nchunks) c1 = nchunks;
    // 11 haloed fields read; 25 FP64, 25 FP32, 25 difference-form FP32 (and
    // 25 BF16) planes, fcscal and 1 / fcscal written per cell
    {
        const double cells = (double)h->d.n * (c1 - c0) / nchunks;
        ProfScope ps(h, PCF_PROF_ASSEMBLE, (11.0 * 8 + 25.0 * 16 + (h->coef16 ? 25.0 * 2 : 0.0) + 12.0) * cells);
        int rc = pcf_launch_assemble(h, dt, rf, damp_h, c0, c1);
        if (rc) return rc;
    }
    if (c1 == nchunks) {
        h->operator_set = 1;
        h->op_version += 1;
    }
    return PCF_OK;
}

static int assemble_device(pcf_handle *h, double dt, double rf, int damp_h) {
    if (!h->grid_set || !h->background_set) return PCF_ENOTREADY;
    return assemble_chunks(h, dt, rf, damp_h, 0, -1);
}

int pcf_compute_operator(pcf_handle *h, const double *rho, const double *betar, const double *p, double dt,
                         double rayleigh_factor, int damp_h, double *coef) {
    if (!h || !rho || !betar) return PCF_EINVAL;
    if (h->dims.model == PCF_MODEL_COMPRESSIBLE && !p) return PCF_EINVAL;
    if (dt == 0.0) return PCF_EINVAL;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    const size_t b = sizeof(double) * (size_t)h->nh;
    PCF_CUDA_TRY(cudaMemcpyAsync(h->rho, rho, b, cudaMemcpyHostToDevice, h->stream));
    PCF_CUDA_TRY(cudaMemcpyAsync(h->betar, betar, b, cudaMemcpyHostToDevice, h->stream));
    if (p) PCF_CUDA_TRY(cudaMemcpyAsync(h->p, p, b, cudaMemcpyHostToDevice, h->stream));
    int rc = assemble_device(h, dt, rayleigh_factor, damp_h);
    if (rc) return rc;
    if (coef)
        PCF_CUDA_TRY(cudaMemcpyAsync(coef, h->coef64, sizeof(double) * h->d.n * PCF_NCOEF, cudaMemcpyDeviceToHost,
                                     h->stream));
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return PCF_OK;
}

int pcf_set_operator(pcf_handle *h, const double *coef) {
    if (!h || !coef) return PCF_EINVAL;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    const long long m = h->d.n * PCF_NCOEF;
    PCF_CUDA_TRY(cudaMemcpyAsync(h->coef64, coef, sizeof(double) * m, cudaMemcpyHostToDevice, h->stream));
    k_coef_to_float<<<vec_grid(m), 256, 0, h->stream>>>(h->coef64, h->coef32, m);
    h->launches += 1;
    PCF_CUDA_TRY(cudaGetLastError());
    if (h->coef16) {
        k_float_to_bf16<<<vec_grid(m), 256, 0, h->stream>>>(h->coef32, h->coef16, m);
        h->launches += 1;
        PCF_CUDA_TRY(cudaGetLastError());
    }
    h->operator_set = 1;
    h->op_version += 1;
    h->fac_deta = std::nan("");
    int rc = build_diff(h, h->background_set);
    if (rc) return rc;
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return PCF_OK;
}

// Upload an interior vector into d64 and, for FP32, a rounded copy into d32.
static int upload_vec(pcf_handle *h, const double *src, double *d64, float *d32) {
    PCF_CUDA_TRY(cudaMemcpyAsync(d64, src, sizeof(double) * h->d.n, cudaMemcpyHostToDevice, h->stream));
    if (d32) {
        k_to_float<<<vec_grid(h->d.n), 256, 0, h->stream>>>(d64, d32, h->d.n, 1.0);
        PCF_CUDA_TRY(cudaGetLastError());
    }
    return PCF_OK;
}

int pcf_apply_operator(pcf_handle *h, const double *sin_, double *ls, int mode, int precision) {
    if (!h || !sin_ || !ls || (mode != PCF_TOTAL && mode != PCF_HORIZONTAL)) return PCF_EINVAL;
    if (!h->operator_set) return PCF_ENOTREADY;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    int rc;
    if (precision == PCF_PRECISION_MIXED) {
        // the FP32 difference-form operator of the mixed solve, applied to s
        if (mode != PCF_TOTAL) return PCF_EINVAL;
        if ((rc = upload_vec(h, sin_, h->b64, nullptr))) return rc;
        k_to_pi<<<vec_grid(h->d.n), 256, 0, h->stream>>>(h->b64, h->rfc32, h->s32, h->d.n);
        h->launches += 1;
        PCF_CUDA_TRY(cudaGetLastError());
        StencilArgs<float> a;
        a.coef = h->coefB32;
        a.s = h->s32;
        a.out = h->t32;
        a.w1 = nullptr;
        a.deta = 0;
        if ((rc = launch_stencil<float, false, EPI_STORE, true>(h, a))) return rc;
        k_to_double<<<vec_grid(h->d.n), 256, 0, h->stream>>>(h->t32, h->w64, h->d.n);
        h->launches += 1;
        PCF_CUDA_TRY(cudaGetLastError());
    } else if (precision == PCF_PRECISION_FP32) {
        if ((rc = upload_vec(h, sin_, h->b64, h->s32))) return rc;
        StencilArgs<float> a;
        a.coef = h->coef32;
        a.s = h->s32;
        a.out = h->t32;
        a.w1 = nullptr;
        a.deta = 0;
        a.guard = nullptr;
        rc = mode == PCF_TOTAL ? launch_stencil<float, false, EPI_STORE>(h, a)
                               : launch_stencil<float, true, EPI_STORE>(h, a);
        if (rc) return rc;
        k_to_double<<<vec_grid(h->d.n), 256, 0, h->stream>>>(h->t32, h->w64, h->d.n);
        PCF_CUDA_TRY(cudaGetLastError());
    } else {
        if ((rc = upload_vec(h, sin_, h->b64, nullptr))) return rc;
        StencilArgs<double> a;
        a.coef = h->coef64;
        a.s = h->b64;
        a.out = h->w64;
        a.w1 = nullptr;
        a.deta = 0;
        a.guard = nullptr;
        rc = mode == PCF_TOTAL ? launch_stencil<double, false, EPI_STORE>(h, a)
                               : launch_stencil<double, true, EPI_STORE>(h, a);
        if (rc) return rc;
    }
    PCF_CUDA_TRY(cudaMemcpyAsync(ls, h->w64, sizeof(double) * h->d.n, cudaMemcpyDeviceToHost, h->stream));
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return PCF_OK;
}

int pcf_apply_preconditioner(pcf_handle *h, const double *sin_, double *sout, const pcf_params *prm, int precision) {
    if (!h || !sin_ || !sout || !prm || prm->preconditioner_iterations < 1) return PCF_EINVAL;
    if (!h->operator_set) return PCF_ENOTREADY;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    const double deta = deta_of(h, prm->dtau);
    int rc = ensure_factors(h, deta);
    if (rc) return rc;
    if (precision == PCF_PRECISION_FP32) {
        if ((rc = upload_vec(h, sin_, h->b64, h->s32))) return rc;
        float *z = nullptr;
        rc = precond_apply<float, TH_B>(h, work32(h), h->s32, prm->preconditioner_iterations, deta, nullptr, &z);
        if (rc) return rc;
        k_to_double<<<vec_grid(h->d.n), 256, 0, h->stream>>>(z, h->w64, h->d.n);
        PCF_CUDA_TRY(cudaGetLastError());
    } else {
        if ((rc = upload_vec(h, sin_, h->s64, nullptr))) return rc;
        double *z = nullptr;
        rc = precond_apply<double, TH_B>(h, work64(h), h->s64, prm->preconditioner_iterations, deta, nullptr, &z);
        if (rc) return rc;
        PCF_CUDA_TRY(cudaMemcpyAsync(h->w64, z, sizeof(double) * h->d.n, cudaMemcpyDeviceToDevice, h->stream));
    }
    PCF_CUDA_TRY(cudaMemcpyAsync(sout, h->w64, sizeof(double) * h->d.n, cudaMemcpyDeviceToHost, h->stream));
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return PCF_OK;
}

int pcf_multigrid_levels(pcf_handle *h, const pcf_params *prm, int cap, int *nlevels, int *dims) {
    if (!h || !prm || !nlevels || cap < 0 || (cap > 0 && !dims)) return PCF_EINVAL;
    if (!h->operator_set) return PCF_ENOTREADY;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    int rc = mg_prepare(h, prm);
    if (rc) return rc;
    const int nl = (int)h->mg->lv.size();
    *nlevels = nl;
    for (int l = 0; l < nl && l < cap; ++l) {
        dims[3 * l] = h->mg->lv[l].d.nx;
        dims[3 * l + 1] = h->mg->lv[l].d.ny;
        dims[3 * l + 2] = h->mg->lv[l].d.nz;
    }
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return PCF_OK;
}

int pcf_multigrid_operator(pcf_handle *h, int level, double *coef) {
    if (!h || !coef || !h->mg || level < 0 || level >= (int)h->mg->lv.size()) return PCF_EINVAL;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    const MgLevel &L = h->mg->lv[level];
    const long long m = L.d.n * PCF_NCOEF;
    if (level == 0) {
        PCF_CUDA_TRY(cudaMemcpyAsync(coef, h->coef64, sizeof(double) * m, cudaMemcpyDeviceToHost, h->stream));
        PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
        return PCF_OK;
    }
    std::vector<float> tmp((size_t)m);
    PCF_CUDA_TRY(cudaMemcpyAsync(tmp.data(), L.coef, sizeof(float) * m, cudaMemcpyDeviceToHost, h->stream));
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    for (long long q = 0; q < m; ++q) coef[q] = (double)tmp[(size_t)q];
    return PCF_OK;
}

int pcf_apply_multigrid(pcf_handle *h, const double *sin_, double *sout, const pcf_params *prm) {
    if (!h || !sin_ || !sout || !prm) return PCF_EINVAL;
    if (!h->operator_set) return PCF_ENOTREADY;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    int rc = mg_prepare(h, prm);
    if (rc) return rc;
    if ((rc = upload_vec(h, sin_, h->b64, h->s32))) return rc;
    float *z = nullptr;
    rc = mg_precond<TH_B>(h, work32(h), h->s32, nullptr, &z, h->za32, h->zb32, nullptr);
    if (rc) return rc;
    k_to_double<<<vec_grid(h->d.n), 256, 0, h->stream>>>(z, h->w64, h->d.n);
    PCF_CUDA_TRY(cudaGetLastError());
    PCF_CUDA_TRY(cudaMemcpyAsync(sout, h->w64, sizeof(double) * h->d.n, cudaMemcpyDeviceToHost, h->stream));
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return PCF_OK;
}

int pcf_autotune_entries(pcf_tune_entry *out, int cap, int *count) {
    if (!count || cap < 0 || (cap > 0 && !out)) return PCF_EINVAL;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    *count = (int)g_tune.size();
    for (int q = 0; q < cap && q < (int)g_tune.size(); ++q) out[q] = g_tune[q].e;
    return PCF_OK;
}

int pcf_autotune_clear(void) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune.clear();
    return PCF_OK;
}

// Staging for the host-array entry points of the winds (allocated once).
static int ensure_stage(pcf_handle *h) {
    if (h->stage) return PCF_OK;
    return dalloc(h, (void **)&h->stage, 6 * sizeof(double) * (size_t)h->nh);
}

// compute_lhs! on device arrays.
static int compute_lhs_device(pcf_handle *h, const double *d_u, const double *d_v, const double *d_w,
                              const double *d_heat, double *d_rhs, double *tolref) {
    if (!h->grid_set || !h->background_set) return PCF_ENOTREADY;
    LhsArgs a;
    a.nx = h->d.nx;
    a.ny = h->d.ny;
    a.nz = h->d.nz;
    a.nxx = h->nxx;
    a.nyy = h->nyy;
    a.nbx = h->dims.nbx;
    a.nby = h->dims.nby;
    a.nbz = h->dims.nbz;
    a.compressible = h->dims.model == PCF_MODEL_COMPRESSIBLE;
    a.rdx = 1.0 / h->dx;
    a.rdy = 1.0 / h->dy;
    a.rdz = 1.0 / h->dz;
    // Ma^2 kappa: Ma = uref / aref = 1 (Constants.jl:124, :149), kappa = (gamma - 1) / gamma (:115)
    a.c = 1.0 * 1.0 * ((1.4 - 1.0) / 1.4);
    a.jac = h->jac;
    a.pbar = h->pbar;
    a.rfch = h->rfch;
    a.u = d_u;
    a.v = d_v;
    a.w = d_w;
    a.heating = d_heat;
    a.rhs = d_rhs;
    a.red = red(h, nullptr, FIN_STORE, h->dot_out);
    {
        ProfScope ps(h, PCF_PROF_ASSEMBLE, (a.compressible ? 10.0 : 14.0) * 8 * (double)h->d.n);
        k_compute_lhs<<<vec_grid(h->d.n), 256, 0, h->stream>>>(a);
        PCF_CUDA_TRY(cudaGetLastError());
    }
    double sums[2] = {0, 0};
    PCF_CUDA_TRY(cudaMemcpyAsync(sums, h->dot_out, sizeof(sums), cudaMemcpyDeviceToHost, h->stream));
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    // compute_lhs!.jl:138-157 (one rank: x_size y_size z_size = nx ny nz)
    const double nn = (double)h->d.n;
    const double divl2 = std::sqrt(sums[0] / nn), norm = std::sqrt(sums[1] / nn);
    if (!std::isfinite(divl2) || !std::isfinite(norm)) return PCF_ENONFINITE;
    if (norm != 0.0)
        *tolref = divl2 / norm;
    else if (divl2 == 0.0)
        *tolref = 1.0;
    else
        return PCF_ENONFINITE;  // the reference raises "divl2_norm = 0 while divl2 != 0"
    return PCF_OK;
}

int pcf_compute_lhs_device(pcf_handle *h, const double *d_u, const double *d_v, const double *d_w,
                           const double *d_heating, double *d_rhs, double *tolref) {
    if (!h || !d_u || !d_v || !d_w || !d_rhs || !tolref) return PCF_EINVAL;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    return compute_lhs_device(h, d_u, d_v, d_w, d_heating, d_rhs, tolref);
}

int pcf_compute_lhs(pcf_handle *h, const double *u, const double *v, const double *w, const double *heating,
                    double *rhs, double *tolref) {
    if (!h || !u || !v || !w || !rhs || !tolref) return PCF_EINVAL;
    if (!h->grid_set || !h->background_set) return PCF_ENOTREADY;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    int rc0 = ensure_stage(h);
    if (rc0) return rc0;
    const size_t hb = sizeof(double) * (size_t)h->nh;
    double *du = h->stage, *dv = h->stage + h->nh, *dw = h->stage + 2 * h->nh;
    PCF_CUDA_TRY(cudaMemcpyAsync(du, u, hb, cudaMemcpyHostToDevice, h->stream));
    PCF_CUDA_TRY(cudaMemcpyAsync(dv, v, hb, cudaMemcpyHostToDevice, h->stream));
    PCF_CUDA_TRY(cudaMemcpyAsync(dw, w, hb, cudaMemcpyHostToDevice, h->stream));
    if (heating)
        PCF_CUDA_TRY(cudaMemcpyAsync(h->t64, heating, sizeof(double) * h->d.n, cudaMemcpyHostToDevice, h->stream));
    int rc = compute_lhs_device(h, du, dv, dw, heating ? h->t64 : nullptr, h->s64, tolref);
    if (rc) return rc;
    PCF_CUDA_TRY(cudaMemcpyAsync(rhs, h->s64, sizeof(double) * h->d.n, cudaMemcpyDeviceToHost, h->stream));
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return PCF_OK;
}

// Algorithmic bytes of the predictor (each field a kernel touches read or
// written once per point): the U/V kernel reads u, v, pip, rho, rhobar,
// pbar, met13, met23 (+ betar with damping, jac and p when Compressible,
// dudt or dvdt with WKB) and writes u, v, and copies w to wold over the
// haloed grid; the W and RhoP kernels read 14 fields each (+ thetabar and p,
// + dudt and dvdt) and write one; each of the two boundary fills reads and
// writes the ghost cells of the model's 5-7 predictands.
static double predictor_bytes(const pcf_handle *h, int damp, bool wkb) {
    const bool comp = h->dims.model == PCF_MODEL_COMPRESSIBLE;
    const double n = (double)h->d.n, nh = (double)h->nh;
    const int extra = (comp ? 2 : 0) + (wkb ? 2 : 0);
    const double uv = 8 + (damp ? 1 : 0) + extra + 2, w = 14 + extra + 1, rp = 14 + extra + 1;
    const int nf = h->dims.model == PCF_MODEL_BOUSSINESQ ? 5 : (comp ? 7 : 6);
    return 8.0 * (n * (uv + w + rp) + 2.0 * nh + 2.0 * 2.0 * nf * (nh - n));
}

// Algorithmic bytes of the corrector: the dpip fill (ghost cells read and
// written), the U/V kernel (dpip, rho, rhobar, pbar, met13, met23, u, v read
// (+ betar, + jac and p), u, v, corx, cory written) and the W/RhoP/PiP kernel
// (15 fields read (+ thetabar, p), w, rhop, pip written).
static double corrector_bytes(const pcf_handle *h, int damp) {
    const bool comp = h->dims.model == PCF_MODEL_COMPRESSIBLE;
    const double n = (double)h->d.n, nh = (double)h->nh;
    return 8.0 * (2.0 * (nh - n) + n * (8 + (damp ? 1 : 0) + (comp ? 2 : 0) + 4) + n * (15 + (comp ? 2 : 0) + 3));
}

int pcf_correct_device(pcf_handle *h, double dt, double rayleigh_factor, int damp_horizontal_wind_on_rhs,
                       double *d_dpip, double *d_u, double *d_v, double *d_w, double *d_rhop, double *d_pip) {
    if (!h || !d_dpip || !d_u || !d_v || !d_w || !d_rhop || !d_pip) return PCF_EINVAL;
    if (!h->grid_set || !h->background_set) return PCF_ENOTREADY;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    if (!h->corr) {
        int rc = dalloc(h, (void **)&h->corr, 2 * sizeof(double) * (size_t)h->nh);
        if (rc) return rc;
    }
    int rc;
    {
        ProfScope ps(h, PCF_PROF_CORRECT, corrector_bytes(h, damp_horizontal_wind_on_rhs), 0);
        rc = pcf_launch_correct(h, dt, rayleigh_factor, damp_horizontal_wind_on_rhs, d_dpip, d_u, d_v, d_w, d_rhop,
                                d_pip, h->corr, h->corr + h->nh);
    }
    if (rc) return rc;
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    prof_flush(h, 0);
    return PCF_OK;
}

int pcf_correct(pcf_handle *h, double dt, double rayleigh_factor, int damp_horizontal_wind_on_rhs, double *dpip,
                double *u, double *v, double *w, double *rhop, double *pip) {
    if (!h || !dpip || !u || !v || !w || !rhop || !pip) return PCF_EINVAL;
    if (!h->grid_set || !h->background_set) return PCF_ENOTREADY;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    int rc = ensure_stage(h);
    if (rc) return rc;
    double *host[6] = {dpip, u, v, w, rhop, pip};
    const size_t hb = sizeof(double) * (size_t)h->nh;
    for (int q = 0; q < 6; ++q)
        PCF_CUDA_TRY(cudaMemcpyAsync(h->stage + q * h->nh, host[q], hb, cudaMemcpyHostToDevice, h->stream));
    double *s = h->stage;
    const long long nh = h->nh;
    if ((rc = pcf_correct_device(h, dt, rayleigh_factor, damp_horizontal_wind_on_rhs, s, s + nh, s + 2 * nh,
                                 s + 3 * nh, s + 4 * nh, s + 5 * nh)))
        return rc;
    for (int q = 0; q < 6; ++q)
        PCF_CUDA_TRY(cudaMemcpyAsync(host[q], h->stage + q * h->nh, hb, cudaMemcpyDeviceToHost, h->stream));
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return PCF_OK;
}

int pcf_apply_corrector_device(pcf_handle *h, double *d_u, double *d_v, double *d_w, const double *d_rho,
                               double *d_rhop, const double *d_betar, const double *d_p, double *d_pip,
                               const double *d_heating, double dt, double rayleigh_factor, const pcf_params *prm,
                               double *d_dpip, pcf_result *res) {
    if (!h || !d_u || !d_v || !d_w || !d_rho || !d_rhop || !d_betar || !d_pip || !prm || !d_dpip || !res)
        return PCF_EINVAL;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    NvtxScope r("pcf_apply_corrector_device");
    // apply_corrector!.jl:44-61: compute_lhs!, solve_poisson!, dpip halos, correct!
    double tolref = 0;
    int rc = compute_lhs_device(h, d_u, d_v, d_w, d_heating, h->s64, &tolref);
    if (rc) return rc;
    if ((rc = pcf_solve_device(h, h->s64, d_rho, d_betar, d_p, dt, rayleigh_factor, tolref, prm, d_dpip, res)))
        return rc;
    if (res->errflag) return PCF_OK;  // the reference returns (errflag, niter) uncorrected
    return pcf_correct_device(h, dt, rayleigh_factor, prm->damp_horizontal_wind_on_rhs, d_dpip, d_u, d_v, d_w,
                              d_rhop, d_pip);
}

// ------------------------------------------------- implicit half step --

static int predictor_ready(pcf_handle *h, const void *u, const void *v, const void *w, const void *rho,
                           const void *rhop, const void *pip, const void *p, const void *betar, const void *dudt,
                           const void *dvdt) {
    if (!h || !u || !v || !w || !rho || !rhop || !pip || !betar) return PCF_EINVAL;
    if ((dudt == nullptr) != (dvdt == nullptr)) return PCF_EINVAL;
    if (h->dims.model == PCF_MODEL_COMPRESSIBLE && !p) return PCF_EINVAL;
    // the wall reflections read interior levels only; W lives on nz - 1 levels
    if (h->d.nz <= h->dims.nbz || h->d.nz < 2) return PCF_EINVAL;
    if (!h->grid_set || !h->background_set) return PCF_ENOTREADY;
    return PCF_OK;
}

int pcf_set_predictand_boundaries_device(pcf_handle *h, double *d_rho, double *d_rhop, double *d_u, double *d_v,
                                         double *d_w, double *d_pip, double *d_p) {
    if (!h || !d_rhop || !d_u || !d_v || !d_w || !d_pip) return PCF_EINVAL;
    if (h->dims.model != PCF_MODEL_BOUSSINESQ && !d_rho) return PCF_EINVAL;
    if (h->dims.model == PCF_MODEL_COMPRESSIBLE && !d_p) return PCF_EINVAL;
    if (h->d.nz <= h->dims.nbz) return PCF_EINVAL;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    int rc = pcf_launch_fill_predictands(h, d_rho, d_rhop, d_u, d_v, d_w, d_pip, d_p);
    if (rc) return rc;
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return PCF_OK;
}

int pcf_modify_compressible_wind_device(pcf_handle *h, const double *d_p, double *d_u, double *d_v, double *d_w,
                                        int divide) {
    if (!h || !d_u || !d_v || !d_w) return PCF_EINVAL;
    if (h->dims.model == PCF_MODEL_COMPRESSIBLE && !d_p) return PCF_EINVAL;
    if (!h->grid_set) return PCF_ENOTREADY;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    int rc = pcf_launch_modify_wind(h, d_p, d_u, d_v, d_w, divide);
    if (rc) return rc;
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return PCF_OK;
}

static double *wold_scratch(pcf_handle *h, double *d_wold, int *rc) {
    *rc = PCF_OK;
    if (d_wold) return d_wold;
    if (!h->corr) *rc = dalloc(h, (void **)&h->corr, 2 * sizeof(double) * (size_t)h->nh);
    return h->corr;  // consumed by the RhoP update before the corrector reuses it
}

int pcf_implicit_predictor_device(pcf_handle *h, double dt, double rayleigh_factor, int damp_horizontal_wind_on_rhs,
                                  double *d_u, double *d_v, double *d_w, double *d_rho, double *d_rhop,
                                  double *d_pip, double *d_p, const double *d_betar, const double *d_dudt,
                                  const double *d_dvdt, double *d_wold) {
    int rc = predictor_ready(h, d_u, d_v, d_w, d_rho, d_rhop, d_pip, d_p, d_betar, d_dudt, d_dvdt);
    if (rc) return rc;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    double *wold = wold_scratch(h, d_wold, &rc);
    if (rc) return rc;
    {
        ProfScope ps(h, PCF_PROF_PREDICT, predictor_bytes(h, damp_horizontal_wind_on_rhs, d_dudt != nullptr), 0);
        if ((rc = pcf_launch_predictor(h, dt, rayleigh_factor, damp_horizontal_wind_on_rhs, d_u, d_v, d_w, d_rho,
                                       d_rhop, d_pip, d_p, d_betar, d_dudt, d_dvdt, wold)))
            return rc;
    }
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    prof_flush(h, 0);
    return PCF_OK;
}

int pcf_implicit_step_device(pcf_handle *h, double dt, double rayleigh_factor, const pcf_params *prm, double *d_u,
                             double *d_v, double *d_w, double *d_rho, double *d_rhop, double *d_pip, double *d_p,
                             const double *d_betar, const double *d_dudt, const double *d_dvdt,
                             const double *d_heating, double *d_wold, double *d_dpip, pcf_result *res) {
    int rc = predictor_ready(h, d_u, d_v, d_w, d_rho, d_rhop, d_pip, d_p, d_betar, d_dudt, d_dvdt);
    if (rc) return rc;
    if (!prm || !d_dpip || !res) return PCF_EINVAL;
    if (dt == 0.0) return PCF_EINVAL;  // solve_poisson!.jl:46-48 raises
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    double *wold = wold_scratch(h, d_wold, &rc);
    if (rc) return rc;
    const int damp = prm->damp_horizontal_wind_on_rhs;
    NvtxScope r("pcf_implicit_step_device");
    cudaEvent_t ev[2] = {nullptr, nullptr};
    PCF_CUDA_TRY(cudaEventCreate(&ev[0]));
    if (cudaEventCreate(&ev[1]) != cudaSuccess) {
        cudaEventDestroy(ev[0]);
        return pcf_set_cuda_error(cudaGetLastError());
    }
    auto body = [&]() -> int {
        PCF_CUDA_TRY(cudaEventRecord(ev[0], h->stream));
        // implicit_integration!.jl:49-63
        int r;
        if ((r = pcf_launch_modify_wind(h, d_p, d_u, d_v, d_w, 0))) return r;
        if ((r = pcf_launch_fill_predictands(h, d_rho, d_rhop, d_u, d_v, d_w, d_pip, d_p))) return r;
        {
            ProfScope ps(h, PCF_PROF_PREDICT, predictor_bytes(h, damp, d_dudt != nullptr), 0);
            if ((r = pcf_launch_predictor(h, dt, rayleigh_factor, damp, d_u, d_v, d_w, d_rho, d_rhop, d_pip, d_p,
                                          d_betar, d_dudt, d_dvdt, wold)))
                return r;
        }
        // :65-71: apply_corrector!; like the reference, an unconverged solve
        // returns with the predicted (uncorrected) fields and errflag set
        if ((r = pcf_apply_corrector_device(h, d_u, d_v, d_w, d_rho, d_rhop, d_betar, d_p, d_pip, d_heating, dt,
                                            rayleigh_factor, prm, d_dpip, res)))
            return r;
        if (!res->errflag) {
            // :75-77
            if ((r = pcf_launch_modify_wind(h, d_p, d_u, d_v, d_w, 1))) return r;
            if ((r = pcf_launch_fill_predictands(h, d_rho, d_rhop, d_u, d_v, d_w, d_pip, d_p))) return r;
        }
        PCF_CUDA_TRY(cudaEventRecord(ev[1], h->stream));
        PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
        float ms = 0;
        PCF_CUDA_TRY(cudaEventElapsedTime(&ms, ev[0], ev[1]));
        res->ms_total = ms;
        prof_flush(h, 0);
        return PCF_OK;
    };
    rc = body();
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    return rc;
}

int pcf_implicit_step(pcf_handle *h, double dt, double rayleigh_factor, const pcf_params *prm, double *u, double *v,
                      double *w, double *rho, double *rhop, double *pip, double *p, const double *betar,
                      const double *dudt, const double *dvdt, const double *heating, double *wold, double *dpip,
                      pcf_result *res) {
    int rc = predictor_ready(h, u, v, w, rho, rhop, pip, p, betar, dudt, dvdt);
    if (rc) return rc;
    if (!prm || !dpip || !res) return PCF_EINVAL;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    const size_t nh = (size_t)h->nh, n = (size_t)h->d.n;
    if (!h->istage && (rc = dalloc(h, (void **)&h->istage, sizeof(double) * (12 * nh + n)))) return rc;
    double *s = h->istage;
    double *d[12];
    for (int q = 0; q < 12; ++q) d[q] = s + q * nh;
    double *d_heat = s + 12 * nh;
    // u v w rho rhop pip p betar dudt dvdt wold dpip
    const double *in[10] = {u, v, w, rho, rhop, pip, p, betar, dudt, dvdt};
    const size_t hb = sizeof(double) * nh;
    for (int q = 0; q < 10; ++q)
        if (in[q]) PCF_CUDA_TRY(cudaMemcpyAsync(d[q], in[q], hb, cudaMemcpyHostToDevice, h->stream));
    PCF_CUDA_TRY(cudaMemcpyAsync(d[11], dpip, hb, cudaMemcpyHostToDevice, h->stream));
    if (heating) PCF_CUDA_TRY(cudaMemcpyAsync(d_heat, heating, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    if ((rc = pcf_implicit_step_device(h, dt, rayleigh_factor, prm, d[0], d[1], d[2], d[3], d[4], d[5], p ? d[6] : nullptr,
                                       d[7], dudt ? d[8] : nullptr, dvdt ? d[9] : nullptr, heating ? d_heat : nullptr,
                                       d[10], d[11], res)))
        return rc;
    double *out[8] = {u, v, w, rho, rhop, pip, p, dpip};
    const int idx[8] = {0, 1, 2, 3, 4, 5, 6, 11};
    for (int q = 0; q < 8; ++q)
        if (out[q]) PCF_CUDA_TRY(cudaMemcpyAsync(out[q], d[idx[q]], hb, cudaMemcpyDeviceToHost, h->stream));
    if (wold) PCF_CUDA_TRY(cudaMemcpyAsync(wold, d[10], hb, cudaMemcpyDeviceToHost, h->stream));
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return PCF_OK;
}

int pcf_global_dot(pcf_handle *h, const double *a, const double *b, double *out) {
    if (!h || !a || !b || !out) return PCF_EINVAL;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    PCF_CUDA_TRY(cudaMemcpyAsync(h->s64, a, sizeof(double) * h->d.n, cudaMemcpyHostToDevice, h->stream));
    PCF_CUDA_TRY(cudaMemcpyAsync(h->t64, b, sizeof(double) * h->d.n, cudaMemcpyHostToDevice, h->stream));
    k_dot<double><<<vec_grid(h->d.n), 256, 0, h->stream>>>(h->s64, h->t64, h->d.n, red(h, nullptr, FIN_STORE, h->dot_out));
    PCF_CUDA_TRY(cudaGetLastError());
    PCF_CUDA_TRY(cudaMemcpyAsync(out, h->dot_out, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    return PCF_OK;
}

// FP64 true residual r = b - A x (into r64) and its RMS.
static int true_residual(pcf_handle *h, const double *b, const double *x, double *rms) {
    StencilArgs<double> a;
    a.coef = h->coef64;
    a.s = x;
    a.out = h->w64;
    a.w1 = b;
    a.deta = 0;
    a.guard = nullptr;
    a.red = red(h, nullptr, FIN_STORE, h->dot_out);
    int rc = launch_stencil<double, false, EPI_RESID>(h, a);
    if (rc) return rc;
    double rr = 0;
    PCF_CUDA_TRY(cudaMemcpyAsync(&rr, h->dot_out, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    *rms = std::sqrt(rr / (double)h->d.n);
    return PCF_OK;
}

// The FP64 residual of the zero initial guess, r64 = b (into w64, as
// true_residual leaves it), and its RMS: one pass over b instead of an
// operator apply.
static int zero_guess_residual(pcf_handle *h, const double *b, double *rms) {
    k_copy_sumsq<<<vec_grid(h->d.n), 256, 0, h->stream>>>(b, h->w64, h->d.n, red(h, nullptr, FIN_STORE, h->dot_out));
    h->launches += 1;
    PCF_CUDA_TRY(cudaGetLastError());
    double rr = 0;
    PCF_CUDA_TRY(cudaMemcpyAsync(&rr, h->dot_out, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    *rms = std::sqrt(rr / (double)h->d.n);
    return PCF_OK;
}

// Grids of at most kTinyMaxCells cells: the reference FP64 BiCGSTAB in one
// thread block (pcf_tiny.cuh), whatever the precision and multigrid settings
// (on such grids the solve is bound by launch latency, so neither reduced
// precision nor the multigrid hierarchy pays off).  Convergence is tested on
// the recursive residual as in the reference; the FP64 true residual is
// reported and, for the mixed precision or true-residual settings, decides
// errflag.
static int tiny_solve(pcf_handle *h, double tol, const pcf_params *prm, const double **xres, pcf_result *res) {
    const double deta = deta_of(h, prm->dtau);
    int rc;
    if (prm->preconditioner && (rc = ensure_factors(h, deta))) return rc;
    static int attr_device = -1;
    const size_t smem = sizeof(double) * kTinyVectors * (size_t)h->d.n;
    if (attr_device != h->dims.device) {
        PCF_CUDA_TRY(cudaFuncSetAttribute(k_tiny_bicgstab, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)(sizeof(double) * kTinyVectors * kTinyMaxCells)));
        attr_device = h->dims.device;
    }
    TinyArgs a;
    a.nx = h->d.nx;
    a.ny = h->d.ny;
    a.nz = h->d.nz;
    a.n = (int)h->d.n;
    a.plane = h->d.plane;
    a.coef = h->coef64;
    a.fac = h->fac64;
    a.b = h->b64;
    a.x = h->x64;
    a.tol = tol;
    a.maxit = prm->poisson_iterations;
    a.precond = prm->preconditioner;
    a.pc_iters = prm->preconditioner_iterations;
    a.deta = deta;
    a.scal = h->scal64;
    a.hist = h->hist;
    a.hist_cap = kHistCap;
    {
        ProfScope ps(h, PCF_PROF_APPLY64, 0.0);
        k_tiny_bicgstab<<<1, kTinyThreads, smem, h->stream>>>(a);
        PCF_CUDA_TRY(cudaGetLastError());
    }
    PCF_CUDA_TRY(cudaMemcpyAsync(h->h_scal, h->scal64, sizeof(KrylovScalars), cudaMemcpyDeviceToHost, h->stream));
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    const KrylovScalars ks = *h->h_scal;
    prof_flush(h, 0);
    h->hist_len = std::min(ks.iter, kHistCap);
    res->niter = ks.iter;
    res->nrefine = 0;
    res->status = ks.status;
    res->errflag = ks.converged ? 0 : 1;
    res->b_norm = ks.b_norm;
    res->residual = ks.b_norm > 0 ? ks.res / ks.b_norm : 0.0;
    *xres = h->x64;
    double tr = 0;
    if ((rc = true_residual(h, h->b64, h->x64, &tr))) return rc;
    res->true_residual = ks.b_norm > 0 ? tr / ks.b_norm : 0.0;
    const bool true_test = prm->residual == PCF_RESIDUAL_TRUE || prm->precision == PCF_PRECISION_MIXED;
    if (prm->precision == PCF_PRECISION_MIXED) res->residual = res->true_residual;
    if (true_test && !res->errflag && res->true_residual > tol) res->errflag = 1;
    return PCF_OK;
}

// Iterations the mixed solve gives the learned preconditioner stage to
// converge; a stage that has not by then (the multigrid alone takes 11-16 on
// the benchmark grids) is dropped like one that breaks down.
constexpr int kStageIterations = 60;

// Solves A x = b64 (device) according to prm; the solution ends in *xres
// (a device FP64 buffer owned by the handle).
static int krylov_solve(pcf_handle *h, double tolref, const pcf_params *prm, const double **xres, pcf_result *res) {
    const double tol = prm->tolerance_is_relative ? prm->tolerance : prm->tolerance / tolref;  // :49-53
    LoopCfg c;
    c.precond = prm->preconditioner;
    c.pc_iters = prm->preconditioner_iterations;
    c.deta = deta_of(h, prm->dtau);
    c.flex = 0;
    c.reliable = 0;
    if (c.precond && c.pc_iters < 1) return PCF_EINVAL;
    // the multigrid preconditioner runs in the FP32 loop of the mixed solve only
    if (prm->multigrid && (prm->precision != PCF_PRECISION_MIXED || !c.precond)) return PCF_EINVAL;
    if (h->d.n <= kTinyMaxCells) return tiny_solve(h, tol, prm, xres, res);
    int rc;
    // (the multigrid mixed solve builds the pivots of its own d_eta in mg_prepare)
    if (c.precond && !prm->multigrid && (rc = ensure_factors(h, c.deta))) return rc;
    const int maxit = prm->poisson_iterations;

    if (prm->precision != PCF_PRECISION_MIXED) {
        if (prm->autotune && (rc = autotune_handle(h, prm))) return rc;
        double *x = nullptr;
        RunOut ro;
        rc = bicgstab_run<double>(h, work64(h), h->b64, tol, maxit, c, prm->check_interval, false, &x, &ro);
        if (rc) return rc;
        res->niter = ro.iters;
        res->nrefine = 0;
        res->status = ro.status;
        res->errflag = ro.converged ? 0 : 1;
        res->residual = ro.res;
        res->b_norm = ro.b_norm;
        *xres = x;
        double tr = 0;
        if ((rc = true_residual(h, h->b64, x, &tr))) return rc;
        res->true_residual = ro.b_norm > 0 ? tr / ro.b_norm : 0.0;
        if (prm->residual == PCF_RESIDUAL_TRUE && !res->errflag && res->true_residual > tol) res->errflag = 1;
        return PCF_OK;
    }

    // Mixed precision: FP64 iterative refinement around FP32 BiCGSTAB sweeps.
    // x64 accumulates the correction; r64 = b - A x64 is the FP64 true residual.
    PCF_CUDA_TRY(cudaMemsetAsync(h->x64, 0, sizeof(double) * h->d.n, h->stream));
    double rnorm = 0;
    if ((rc = zero_guess_residual(h, h->b64, &rnorm))) return rc;
    const double b_norm = rnorm;
    res->b_norm = b_norm;
    if ((prm->learned & 1) && h->net && b_norm > 0 && std::isfinite(b_norm)) {
        // learned warm start: x0 = RMS(b) N(b / RMS(b)), then the FP64 residual of x0
        h->launches += 6;
        rc = pcf_net_apply_device(h->net, h->b64, h->d.nx, h->d.ny, h->d.nz, 1.0 / b_norm, b_norm, 0.0, h->x64, 1,
                                  h->stream);
        if (rc) return rc;
        if ((rc = true_residual(h, h->b64, h->x64, &rnorm))) return rc;
    }
    res->niter = 0;
    res->nrefine = 0;
    res->status = PCF_OK;
    res->errflag = 0;
    *xres = h->x64;
    if (!std::isfinite(b_norm)) {
        res->status = PCF_ENONFINITE;
        res->errflag = 1;
        return PCF_OK;
    }
    if (b_norm == 0.0 || 1.0 <= tol) {
        res->residual = 0.0;
        res->true_residual = 0.0;
        return PCF_OK;
    }
    // One FP32 BiCGSTAB iteration on b / RMS(b) with reliable updates: the
    // FP32 correction is folded into x64 and the FP32 residual replaced by the
    // FP64 true residual whenever it fell by inner_tolerance (device-side, see
    // reliable_update).  A breakdown restarts the FP32 iteration from the
    // current FP64 residual (at most max_refinements times).
    Work<float> w = work32_pi(h);
    LoopCfg cm = c;
    cm.flex = 1;
    cm.reliable = 1;
    if (prm->multigrid) {
        if ((rc = mg_prepare(h, prm))) return rc;
        cm.mg = 1;
        cm.deta = h->mg->lv[0].deta;
    }
    if (prm->autotune && (rc = autotune_handle(h, prm))) return rc;
    if ((prm->learned & 2) && h->net && c.precond) {
        if (!h->lr32 && (rc = dalloc(h, (void **)&h->lr32, 2 * sizeof(float) * (size_t)h->d.n))) return rc;
        // one forward outside any graph capture (the GEMM's first launch sets its attributes)
        PCF_CUDA_TRY(cudaMemsetAsync(h->lr32, 0, 2 * sizeof(float) * (size_t)h->d.n, h->stream));
        if ((rc = pcf_net_apply_device(h->net, h->lr32, h->d.nx, h->d.ny, h->d.nz, 1.0, 1.0, 0.0,
                                       h->lr32 + h->d.n, 0, h->stream)))
            return rc;
        cm.learned_pc = 1;
    }
    double rel = rnorm / b_norm;
    int restarts = 0;
    for (;;) {
        k_to_float<<<vec_grid(h->d.n), 256, 0, h->stream>>>(h->w64, w.s, h->d.n, 1.0 / b_norm);
        h->launches += 1;
        PCF_CUDA_TRY(cudaGetLastError());
        float *e = nullptr;
        RunOut ro;
        // with the learned stage the iteration gets kStageIterations to converge
        const int cap = cm.learned_pc ? std::min(maxit - res->niter, kStageIterations) : maxit - res->niter;
        rc = bicgstab_run<float>(h, w, w.s, tol, cap, cm, prm->check_interval, false, &e, &ro, res->niter, 1.0,
                                 b_norm, prm->inner_tolerance, prm->restart_interval);
        if (rc) return rc;
        res->niter += ro.iters;
        res->nrefine += ro.nupdates;
        reliable_bytes(h, ro.nupdates);
        if (ro.nupdates > 0) rel = ro.res;
        if (ro.converged) break;
        const bool stalled = cm.learned_pc && ro.iters >= cap && res->niter < maxit;
        if ((ro.status == PCF_EBREAKDOWN || stalled) && restarts < prm->max_refinements && res->niter < maxit) {
            if (cm.learned_pc) {
                // the plain preconditioner is the fallback: a breakdown, divergence or
                // stall with the learned stage drops the stage for the rest of the solve
                // and discards the FP32 correction since the last reliable update
                // (the FP64 solution keeps every reliable update made with it)
                cm.learned_pc = 0;
            } else {
                // fold what the broken-down iteration accumulated
                k_axpy_f2d<<<vec_grid(h->d.n), 256, 0, h->stream>>>(w.x, h->x64, h->fc64, h->d.n, b_norm);
                h->launches += 1;
                PCF_CUDA_TRY(cudaGetLastError());
            }
            // restart from the true residual
            if ((rc = true_residual(h, h->b64, h->x64, &rnorm))) return rc;
            rel = rnorm / b_norm;
            restarts += 1;
            if (!std::isfinite(rel)) {
                res->status = PCF_ENONFINITE;
                break;
            }
            if (rel <= tol) break;
            continue;
        }
        res->status = ro.status;
        break;
    }
    res->residual = rel;
    res->true_residual = rel;
    res->errflag = rel <= tol ? 0 : 1;
    return PCF_OK;
}

static float elapsed(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

// rhs_ready: an event the solve waits for after the assembly (the right-hand
// side's upload on the copy stream), or null.  assembled: the caller queued
// the assembly (and recorded ev[1] where it starts).
static int solve_common(pcf_handle *h, double dt, double rf, double tolref, const pcf_params *prm, pcf_result *res,
                        const double **x, cudaEvent_t rhs_ready = nullptr, bool assembled = false) {
    // solve_poisson!.jl:52-54
    if (dt == 0.0) return PCF_EINVAL;
    int rc;
    if (!assembled) PCF_CUDA_TRY(cudaEventRecord(h->ev[1], h->stream));
    {
        NvtxScope r("pcf assemble");
        if (!assembled && (rc = assemble_device(h, dt, rf, prm->damp_horizontal_wind_on_rhs))) return rc;
        // the multigrid mixed solve builds the pivots of its own d_eta (mg_prepare)
        const bool mg = prm->multigrid && prm->precision == PCF_PRECISION_MIXED;
        if (prm->preconditioner && !mg && (rc = ensure_factors(h, deta_of(h, prm->dtau)))) return rc;
    }
    if (rhs_ready) PCF_CUDA_TRY(cudaStreamWaitEvent(h->stream, rhs_ready, 0));
    PCF_CUDA_TRY(cudaEventRecord(h->ev[2], h->stream));
    {
        NvtxScope r("pcf krylov");
        if ((rc = krylov_solve(h, tolref, prm, x, res))) return rc;
    }
    PCF_CUDA_TRY(cudaEventRecord(h->ev[3], h->stream));
    return PCF_OK;
}

int pcf_solve(pcf_handle *h, const double *rhs, const double *rho, const double *betar, const double *p, double dt,
              double rayleigh_factor, double tolref, const pcf_params *prm, double *dpip, pcf_result *res) {
    if (!h || !rhs || !rho || !betar || !prm || !dpip || !res) return PCF_EINVAL;
    if (h->dims.model == PCF_MODEL_COMPRESSIBLE && !p) return PCF_EINVAL;
    NvtxScope r("pcf_solve");
    std::memset(res, 0, sizeof(*res));
    if (dt == 0.0) return PCF_EINVAL;
    if (!h->grid_set || !h->background_set) return PCF_ENOTREADY;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    PCF_CUDA_TRY(cudaEventRecord(h->ev[0], h->stream));
    // The assembly's inputs go up in z-slabs on the copy stream (after all
    // earlier work on the handle's stream), and each slab's part of the
    // assembly starts on the handle's stream as soon as the planes it reads
    // are up, so the assembly runs under the remaining uploads.  The
    // right-hand side follows (host-to-device copies share one link, so
    // starting it earlier would only delay them); the Krylov loop, its first
    // reader, waits for it.
    PCF_CUDA_TRY(cudaStreamWaitEvent(h->copy_stream, h->ev[0], 0));
    const int akc = pcf_assemble_chunk_levels();
    const int nchunks = (h->d.nz + akc - 1) / akc;
    const int slabs = std::min(nchunks, (int)(sizeof(h->slab_ev) / sizeof(h->slab_ev[0])));
    const long long plane = (long long)h->nxx * h->nyy, nzz = h->nh / plane;
    long long up = 0;  // haloed z-planes uploaded
    int rc = PCF_OK;
    for (int sl = 0; sl < slabs; ++sl) {
        const int c0 = (int)((long long)nchunks * sl / slabs), c1 = (int)((long long)nchunks * (sl + 1) / slabs);
        // chunk c reads the interior levels up to AKC c1 + 1, haloed plane AKC c1 + 1 + nbz
        const long long end = sl + 1 == slabs ? nzz : std::min(nzz, (long long)akc * c1 + 2 + h->dims.nbz);
        if (end > up) {
            const size_t off = (size_t)(up * plane), cnt = sizeof(double) * (size_t)((end - up) * plane);
            PCF_CUDA_TRY(cudaMemcpyAsync(h->rho + off, rho + off, cnt, cudaMemcpyHostToDevice, h->copy_stream));
            PCF_CUDA_TRY(cudaMemcpyAsync(h->betar + off, betar + off, cnt, cudaMemcpyHostToDevice, h->copy_stream));
            if (p) PCF_CUDA_TRY(cudaMemcpyAsync(h->p + off, p + off, cnt, cudaMemcpyHostToDevice, h->copy_stream));
            up = end;
        }
        PCF_CUDA_TRY(cudaEventRecord(h->slab_ev[sl], h->copy_stream));
        PCF_CUDA_TRY(cudaStreamWaitEvent(h->stream, h->slab_ev[sl], 0));
        if (sl == 0) PCF_CUDA_TRY(cudaEventRecord(h->ev[1], h->stream));
        if ((rc = assemble_chunks(h, dt, rayleigh_factor, prm->damp_horizontal_wind_on_rhs, c0, c1))) break;
    }
    PCF_CUDA_TRY(cudaMemcpyAsync(h->b64, rhs, sizeof(double) * h->d.n, cudaMemcpyHostToDevice, h->copy_stream));
    PCF_CUDA_TRY(cudaEventRecord(h->ev[7], h->copy_stream));
    const double *x = nullptr;
    if (!rc) rc = solve_common(h, dt, rayleigh_factor, tolref, prm, res, &x, h->ev[7], true);
    if (rc) {
        cudaStreamWaitEvent(h->stream, h->ev[7], 0);  // no later call may meet the copy in flight
        return rc;
    }
    if (!res->errflag) {
        k_unscale<<<vec_grid(h->d.n), 256, 0, h->stream>>>(x, h->pbar, h->rhobar, 1.0 / dt, h->d.nx, h->d.ny,
                                                           h->d.nz, h->dims.nbx, h->dims.nby, h->dims.nbz, h->nxx,
                                                           h->nyy, h->w64, 0, 0, 0, h->d.nx, h->d.ny);
        PCF_CUDA_TRY(cudaGetLastError());
        cudaMemcpy3DParms cp;
        std::memset(&cp, 0, sizeof(cp));
        cp.srcPtr = make_cudaPitchedPtr((void *)h->w64, sizeof(double) * h->d.nx, h->d.nx, h->d.ny);
        cp.dstPtr = make_cudaPitchedPtr((void *)dpip, sizeof(double) * h->nxx, h->nxx, h->nyy);
        cp.dstPos = make_cudaPos(sizeof(double) * h->dims.nbx, h->dims.nby, h->dims.nbz);
        cp.extent = make_cudaExtent(sizeof(double) * h->d.nx, h->d.ny, h->d.nz);
        cp.kind = cudaMemcpyDeviceToHost;
        PCF_CUDA_TRY(cudaMemcpy3DAsync(&cp, h->stream));
    }
    PCF_CUDA_TRY(cudaEventRecord(h->ev[4], h->stream));
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    res->ms_upload = elapsed(h->ev[0], h->ev[1]);
    res->ms_assemble = elapsed(h->ev[1], h->ev[2]);
    res->ms_solve = elapsed(h->ev[2], h->ev[3]);
    res->ms_download = elapsed(h->ev[3], h->ev[4]);
    res->ms_total = elapsed(h->ev[0], h->ev[4]);
    prof_flush(h, 0);
    return PCF_OK;
}

int pcf_solve_device(pcf_handle *h, const double *d_rhs, const double *d_rho, const double *d_betar,
                     const double *d_p, double dt, double rayleigh_factor, double tolref, const pcf_params *prm,
                     double *d_dpip, pcf_result *res) {
    if (!h || !d_rhs || !d_rho || !d_betar || !prm || !d_dpip || !res) return PCF_EINVAL;
    if (h->dims.model == PCF_MODEL_COMPRESSIBLE && !d_p) return PCF_EINVAL;
    NvtxScope r("pcf_solve_device");
    std::memset(res, 0, sizeof(*res));
    if (dt == 0.0) return PCF_EINVAL;
    if (!h->grid_set || !h->background_set) return PCF_ENOTREADY;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    const size_t hb = sizeof(double) * (size_t)h->nh;
    PCF_CUDA_TRY(cudaEventRecord(h->ev[0], h->stream));
    PCF_CUDA_TRY(cudaMemcpyAsync(h->rho, d_rho, hb, cudaMemcpyDeviceToDevice, h->stream));
    PCF_CUDA_TRY(cudaMemcpyAsync(h->betar, d_betar, hb, cudaMemcpyDeviceToDevice, h->stream));
    if (d_p) PCF_CUDA_TRY(cudaMemcpyAsync(h->p, d_p, hb, cudaMemcpyDeviceToDevice, h->stream));
    PCF_CUDA_TRY(cudaMemcpyAsync(h->b64, d_rhs, sizeof(double) * h->d.n, cudaMemcpyDeviceToDevice, h->stream));
    const double *x = nullptr;
    int rc = solve_common(h, dt, rayleigh_factor, tolref, prm, res, &x);
    if (rc) return rc;
    if (!res->errflag) {
        k_unscale<<<vec_grid(h->d.n), 256, 0, h->stream>>>(x, h->pbar, h->rhobar, 1.0 / dt, h->d.nx, h->d.ny,
                                                           h->d.nz, h->dims.nbx, h->dims.nby, h->dims.nbz, h->nxx,
                                                           h->nyy, d_dpip, h->dims.nbx, h->dims.nby, h->dims.nbz,
                                                           h->nxx, h->nyy);
        PCF_CUDA_TRY(cudaGetLastError());
    }
    PCF_CUDA_TRY(cudaEventRecord(h->ev[4], h->stream));
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    res->ms_upload = elapsed(h->ev[0], h->ev[1]);
    res->ms_assemble = elapsed(h->ev[1], h->ev[2]);
    res->ms_solve = elapsed(h->ev[2], h->ev[3]);
    res->ms_download = elapsed(h->ev[3], h->ev[4]);
    res->ms_total = elapsed(h->ev[0], h->ev[4]);
    prof_flush(h, 0);
    return PCF_OK;
}

int pcf_bicgstab(pcf_handle *h, const double *rhs, double tolref, const pcf_params *prm, double *solution,
                 pcf_result *res) {
    if (!h || !rhs || !prm || !solution || !res) return PCF_EINVAL;
    std::memset(res, 0, sizeof(*res));
    if (!h->operator_set) return PCF_ENOTREADY;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    PCF_CUDA_TRY(cudaEventRecord(h->ev[0], h->stream));
    PCF_CUDA_TRY(cudaMemcpyAsync(h->b64, rhs, sizeof(double) * h->d.n, cudaMemcpyHostToDevice, h->stream));
    PCF_CUDA_TRY(cudaEventRecord(h->ev[2], h->stream));
    const double *x = nullptr;
    int rc = krylov_solve(h, tolref, prm, &x, res);
    if (rc) return rc;
    PCF_CUDA_TRY(cudaEventRecord(h->ev[3], h->stream));
    PCF_CUDA_TRY(cudaMemcpyAsync(solution, x, sizeof(double) * h->d.n, cudaMemcpyDeviceToHost, h->stream));
    PCF_CUDA_TRY(cudaEventRecord(h->ev[4], h->stream));
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    res->ms_upload = elapsed(h->ev[0], h->ev[2]);
    res->ms_solve = elapsed(h->ev[2], h->ev[3]);
    res->ms_download = elapsed(h->ev[3], h->ev[4]);
    res->ms_total = elapsed(h->ev[0], h->ev[4]);
    prof_flush(h, 0);
    return PCF_OK;
}

long long pcf_launch_count(const pcf_handle *h) { return h ? h->launches : 0; }

int pcf_set_network(pcf_handle *h, pcf_net *net) {
    if (!h) return PCF_EINVAL;
    h->net = net;
    return PCF_OK;
}

extern "C++" {  // the other translation units' records (pcf_assemble.cu, pcf_correct.cu, pcf_net.cu)
unsigned long long pcf_bounds_take_assemble();
unsigned long long pcf_bounds_take_correct();
unsigned long long pcf_bounds_take_net();
}

int pcf_bounds_check_status(int *enabled, long long *site, long long *index) {
    if (!enabled || !site || !index) return PCF_EINVAL;
    *enabled = PCF_BOUNDS_CHECKED;
    *site = 0;
    *index = 0;
    const unsigned long long recs[4] = {pcf_bounds_take_local(), pcf_bounds_take_assemble(),
                                        pcf_bounds_take_correct(), pcf_bounds_take_net()};
    for (unsigned long long r : recs) {
        if (r == ~0ull) return PCF_ECUDA;
        if (r && !*site) {
            *site = (long long)(r >> 40);
            const long long i = (long long)(r & 0xFFFFFFFFFFull);
            *index = i >= (1ll << 39) ? i - (1ll << 40) : i;  // 40-bit two's complement
        }
    }
    return PCF_OK;
}

int pcf_test_stall_staged_copy(pcf_handle *h, int level, double wait_limit_s) {
    if (!h || !(wait_limit_s >= 0.0) || wait_limit_s > 10.0) return PCF_EINVAL;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->test_stall = level >= 0 ? level + 1 : 0;
    h->test_wait_ns = level >= 0 ? (unsigned long long)(wait_limit_s * 1e9) : 0ull;
    if (level >= 0 && h->test_wait_ns == 0) h->test_wait_ns = 1;
    clear_graphs(h);  // captured batches hold the previous setting
    return PCF_OK;
}

int pcf_residual_history(pcf_handle *h, double *out, int cap, int *n) {
    if (!h || !n || (cap > 0 && !out)) return PCF_EINVAL;
    PCF_CUDA_TRY(cudaSetDevice(h->dims.device));
    const int m = std::min(cap, h->hist_len);
    *n = h->hist_len;
    if (m > 0) {
        PCF_CUDA_TRY(cudaMemcpyAsync(out, h->hist, sizeof(double) * m, cudaMemcpyDeviceToHost, h->stream));
        PCF_CUDA_TRY(cudaStreamSynchronize(h->stream));
    }
    return PCF_OK;
}

int pcf_profile_enable(pcf_handle *h, int on) {
    if (!h) return PCF_EINVAL;
    prof_flush(h, 0);
    h->prof_on = on ? 1 : 0;
    for (auto &a : h->prof_acc) a = ProfAcc{0.0, 0, 0.0};
    return PCF_OK;
}

int pcf_profile_read(const pcf_handle *h, int tag, double *ms, long long *count, double *bytes) {
    if (!h || tag < 0 || tag >= PCF_PROF_NTAGS) return PCF_EINVAL;
    if (ms) *ms = h->prof_acc[tag].ms;
    if (count) *count = h->prof_acc[tag].count;
    if (bytes) *bytes = h->prof_acc[tag].bytes;
    return PCF_OK;
}


// ============================================================== ensemble ==
// Mixed-precision solves of several handles (ensemble members, possibly of
// different grid sizes) advanced together: each member's setup runs on its
// own stream, then every batch of check_interval iterations of all members
// is ONE CUDA graph launch (captured once per ensemble and configuration:
// the members' iteration chains are parallel branches forked from and joined
// to the ensemble's stream), and one status read-back per batch serves all
// members.  Members that converge early keep returning at once from their
// kernels (device-side done flag) until the last one finishes.

struct pcf_ensemble {
    std::vector<pcf_handle *> m;
    int device = 0;
    cudaStream_t origin = nullptr;
    cudaEvent_t fork = nullptr, t0 = nullptr, t1 = nullptr, t2 = nullptr, done = nullptr;
    cudaEvent_t slot_ev[2] = {nullptr, nullptr};
    std::vector<cudaEvent_t> join;
    cudaGraphExec_t exec = nullptr;
    long long graph_launches = 0;
    long long launches = 0;
    bool key_valid = false;
    int key_ci = 0, key_precond = 0, key_pc_iters = 0, key_mg = 0, key_mg_ci = 0, key_mg_min = 0, key_maxit = 0;
    double key_dtau = 0, key_mg_dtau = 0;
    KrylovScalars *h_status = nullptr;  // pinned, 2 slots x members
    double *h_norm = nullptr;           // pinned, members
    // the whole solve as one graph launch: a conditional WHILE node around
    // the batch, whose last kernel decides on the device whether to go on
    cudaGraphExec_t loop_exec = nullptr;
    KrylovScalars **d_scal = nullptr;   // device array: every member's FP32 scalars
    int *d_batches = nullptr;           // batches run by the loop (reset before each launch)
};

// Last kernel of the ensemble's loop body: counts the batch and keeps the
// loop going while any member is still iterating and fewer than max_batches
// batches have run.
__global__ void k_ensemble_continue(KrylovScalars *const *scal, int n, int *batches, int max_batches,
                                    cudaGraphConditionalHandle cond) {
    if (threadIdx.x != 0) return;
    const int b = *batches + 1;
    *batches = b;
    bool any = false;
    for (int q = 0; q < n; ++q) any = any || !scal[q]->done;
    cudaGraphSetConditional(cond, (any && b < max_batches) ? 1u : 0u);
}

static LoopCfg ensemble_loop_cfg(pcf_handle *h, const pcf_params *prm) {
    LoopCfg c;
    c.precond = prm->preconditioner;
    c.pc_iters = prm->preconditioner_iterations;
    c.deta = deta_of(h, prm->dtau);
    c.flex = 1;
    c.reliable = 1;
    c.mg = prm->multigrid ? 1 : 0;
    if (c.mg) c.deta = h->mg->lv[0].deta;
    return c;
}

// Records one batch (ci iterations of every member, members as parallel
// branches forked from and joined to the origin stream) into the graph being
// captured on the origin stream; adds the member kernels to *nl.
static int ensemble_record_batch(pcf_ensemble *e, const pcf_params *prm, int ci, long long *nl) {
    std::vector<long long> l0(e->m.size());
    for (size_t q = 0; q < e->m.size(); ++q) l0[q] = e->m[q]->launches;
    int rc = PCF_OK;
    cudaError_t ce = cudaEventRecord(e->fork, e->origin);
    for (size_t q = 0; q < e->m.size() && rc == PCF_OK && ce == cudaSuccess; ++q) {
        pcf_handle *h = e->m[q];
        ce = cudaStreamWaitEvent(h->stream, e->fork, 0);
        if (ce != cudaSuccess) break;
        const LoopCfg c = ensemble_loop_cfg(h, prm);
        const Work<float> w = work32_pi(h);
        for (int it = 0; it < ci && rc == PCF_OK; ++it) rc = bicgstab_iteration<float>(h, w, c);
        if (rc) break;
        ce = cudaEventRecord(e->join[q], h->stream);
        if (ce == cudaSuccess) ce = cudaStreamWaitEvent(e->origin, e->join[q], 0);
    }
    for (size_t q = 0; q < e->m.size(); ++q) {
        *nl += e->m[q]->launches - l0[q];
        e->m[q]->launches = l0[q];  // captured, not launched
    }
    if (rc) return rc;
    return ce == cudaSuccess ? PCF_OK : pcf_set_cuda_error(ce);
}

// The whole iteration as one executable graph: a conditional WHILE node
// whose body is one batch followed by k_ensemble_continue.  Returns PCF_OK
// with e->loop_exec null if the driver has no conditional nodes (the solve
// then launches the batch graph per batch).
static int ensemble_capture_loop(pcf_ensemble *e, const pcf_params *prm, int ci, int max_batches) {
    if (e->loop_exec) {
        cudaGraphExecDestroy(e->loop_exec);
        e->loop_exec = nullptr;
    }
    const int n = (int)e->m.size();
    if (!e->d_scal) {
        PCF_CUDA_TRY(cudaMalloc(&e->d_scal, sizeof(KrylovScalars *) * n));
        PCF_CUDA_TRY(cudaMalloc(&e->d_batches, sizeof(int)));
        std::vector<KrylovScalars *> ptrs(n);
        for (int q = 0; q < n; ++q) ptrs[q] = e->m[q]->scal32;
        PCF_CUDA_TRY(cudaMemcpy(e->d_scal, ptrs.data(), sizeof(KrylovScalars *) * n, cudaMemcpyHostToDevice));
    }
    cudaGraph_t g = nullptr;
    PCF_CUDA_TRY(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle cond;
    cudaGraphNodeParams cp = {};
    cudaGraphNode_t node;
    if (cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault) != cudaSuccess) {
        cudaGetLastError();
        cudaGraphDestroy(g);
        return PCF_OK;
    }
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = cond;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    if (cudaGraphAddNode(&node, g, nullptr, 0, &cp) != cudaSuccess) {
        cudaGetLastError();
        cudaGraphDestroy(g);
        return PCF_OK;
    }
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    cudaError_t ce = cudaStreamBeginCaptureToGraph(e->origin, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (ce != cudaSuccess) {
        cudaGraphDestroy(g);
        return pcf_set_cuda_error(ce);
    }
    long long nl = 0;
    int rc = ensemble_record_batch(e, prm, ci, &nl);
    if (!rc) {
        k_ensemble_continue<<<1, 32, 0, e->origin>>>(e->d_scal, n, e->d_batches, max_batches, cond);
        ce = cudaGetLastError();
    }
    cudaGraph_t out = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(e->origin, &out);
    if (rc || ce != cudaSuccess || ee != cudaSuccess) {
        cudaGraphDestroy(g);
        if (rc) return rc;
        return pcf_set_cuda_error(ce != cudaSuccess ? ce : ee);
    }
    const cudaError_t ei = cudaGraphInstantiate(&e->loop_exec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
        e->loop_exec = nullptr;
        return pcf_set_cuda_error(ei);
    }
    return PCF_OK;
}

static int ensemble_capture(pcf_ensemble *e, const pcf_params *prm, int ci) {
    if (e->exec) {
        cudaGraphExecDestroy(e->exec);
        e->exec = nullptr;
    }
    PCF_CUDA_TRY(cudaStreamBeginCapture(e->origin, cudaStreamCaptureModeThreadLocal));
    long long nl = 0;
    const int rc = ensemble_record_batch(e, prm, ci, &nl);
    cudaGraph_t graph = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(e->origin, &graph);
    if (rc || ee != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        if (rc) return rc;
        return pcf_set_cuda_error(ee);
    }
    const cudaError_t ei = cudaGraphInstantiate(&e->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) return pcf_set_cuda_error(ei);
    e->graph_launches = nl;
    e->key_valid = true;
    e->key_ci = ci;
    e->key_precond = prm->preconditioner;
    e->key_pc_iters = prm->preconditioner_iterations;
    e->key_dtau = prm->dtau;
    e->key_mg = prm->multigrid;
    e->key_mg_ci = prm->mg_coarse_iterations;
    e->key_mg_min = prm->mg_min_columns;
    e->key_mg_dtau = prm->mg_dtau;
    e->key_maxit = prm->poisson_iterations;
    return ensemble_capture_loop(e, prm, ci, (prm->poisson_iterations + ci - 1) / ci);
}

int pcf_ensemble_destroy(pcf_ensemble *e) {
    if (!e) return PCF_OK;
    cudaSetDevice(e->device);
    if (e->exec) cudaGraphExecDestroy(e->exec);
    if (e->loop_exec) cudaGraphExecDestroy(e->loop_exec);
    if (e->d_scal) cudaFree(e->d_scal);
    if (e->d_batches) cudaFree(e->d_batches);
    cudaEvent_t evs[] = {e->fork, e->t0, e->t1, e->t2, e->done, e->slot_ev[0], e->slot_ev[1]};
    for (cudaEvent_t x : evs)
        if (x) cudaEventDestroy(x);
    for (cudaEvent_t x : e->join)
        if (x) cudaEventDestroy(x);
    if (e->h_status) cudaFreeHost(e->h_status);
    if (e->h_norm) cudaFreeHost(e->h_norm);
    if (e->origin) cudaStreamDestroy(e->origin);
    delete e;
    return PCF_OK;
}

int pcf_ensemble_create(pcf_ensemble **out, pcf_handle *const *members, int count) {
    if (!out || !members || count < 1) return PCF_EINVAL;
    *out = nullptr;
    for (int q = 0; q < count; ++q) {
        if (!members[q] || members[q]->dims.device != members[0]->dims.device) return PCF_EINVAL;
        for (int r = 0; r < q; ++r)
            if (members[r] == members[q]) return PCF_EINVAL;  // each member owns its buffers
    }
    PCF_CUDA_TRY(cudaSetDevice(members[0]->dims.device));
    pcf_ensemble *e = new pcf_ensemble();
    e->m.assign(members, members + count);
    e->device = members[0]->dims.device;
    e->join.assign(count, nullptr);
    auto fail = [&](int code) {
        pcf_ensemble_destroy(e);
        return code;
    };
    if (cudaStreamCreateWithFlags(&e->origin, cudaStreamNonBlocking) != cudaSuccess) return fail(PCF_ECUDA);
    cudaEvent_t *evs[] = {&e->fork, &e->t0, &e->t1, &e->t2, &e->done, &e->slot_ev[0], &e->slot_ev[1]};
    for (cudaEvent_t *x : evs)
        if (cudaEventCreate(x) != cudaSuccess) return fail(PCF_ECUDA);
    for (cudaEvent_t &x : e->join)
        if (cudaEventCreateWithFlags(&x, cudaEventDisableTiming) != cudaSuccess) return fail(PCF_ECUDA);
    if (cudaMallocHost((void **)&e->h_status, 2 * sizeof(KrylovScalars) * count) != cudaSuccess) return fail(PCF_ENOMEM);
    if (cudaMallocHost((void **)&e->h_norm, sizeof(double) * count) != cudaSuccess) return fail(PCF_ENOMEM);
    *out = e;
    return PCF_OK;
}

long long pcf_ensemble_launch_count(const pcf_ensemble *e) { return e ? e->launches : 0; }

int pcf_ensemble_solve_device(pcf_ensemble *e, const double *const *d_rhs, const double *const *d_rho,
                              const double *const *d_betar, const double *const *d_p, const double *dt,
                              const double *rayleigh_factor, const double *tolref, const pcf_params *prm,
                              double *const *d_dpip, pcf_result *res) {
    if (!e || !d_rhs || !d_rho || !d_betar || !dt || !rayleigh_factor || !tolref || !prm || !d_dpip || !res)
        return PCF_EINVAL;
    const int n = (int)e->m.size();
    for (int q = 0; q < n; ++q) {
        pcf_handle *h = e->m[q];
        if (!d_rhs[q] || !d_rho[q] || !d_betar[q] || !d_dpip[q] || dt[q] == 0.0) return PCF_EINVAL;
        if (h->dims.model == PCF_MODEL_COMPRESSIBLE && (!d_p || !d_p[q])) return PCF_EINVAL;
        if (!h->grid_set || !h->background_set) return PCF_ENOTREADY;
    }
    // the ensemble advances the mixed-precision iteration only
    if (prm->precision != PCF_PRECISION_MIXED || prm->learned || (prm->preconditioner && prm->preconditioner_iterations < 1) ||
        (prm->multigrid && !prm->preconditioner))
        return PCF_EINVAL;
    PCF_CUDA_TRY(cudaSetDevice(e->device));
    const int ci = prm->check_interval < 1 ? 16 : prm->check_interval;
    const int maxit = prm->poisson_iterations;
    int rc;
    PCF_CUDA_TRY(cudaEventRecord(e->t0, e->origin));
    // setup on every member's stream: inputs, assembly, pivots, multigrid
    // hierarchy, r = b - A 0 in FP64 with its norm read back asynchronously
    for (int q = 0; q < n; ++q) {
        pcf_handle *h = e->m[q];
        std::memset(&res[q], 0, sizeof(pcf_result));
        const size_t hb = sizeof(double) * (size_t)h->nh;
        PCF_CUDA_TRY(cudaStreamWaitEvent(h->stream, e->t0, 0));
        PCF_CUDA_TRY(cudaEventRecord(h->ev[0], h->stream));
        PCF_CUDA_TRY(cudaMemcpyAsync(h->rho, d_rho[q], hb, cudaMemcpyDeviceToDevice, h->stream));
        PCF_CUDA_TRY(cudaMemcpyAsync(h->betar, d_betar[q], hb, cudaMemcpyDeviceToDevice, h->stream));
        if (d_p && d_p[q]) PCF_CUDA_TRY(cudaMemcpyAsync(h->p, d_p[q], hb, cudaMemcpyDeviceToDevice, h->stream));
        PCF_CUDA_TRY(cudaMemcpyAsync(h->b64, d_rhs[q], sizeof(double) * h->d.n, cudaMemcpyDeviceToDevice, h->stream));
        PCF_CUDA_TRY(cudaEventRecord(h->ev[1], h->stream));
        if ((rc = assemble_device(h, dt[q], rayleigh_factor[q], prm->damp_horizontal_wind_on_rhs))) return rc;
        if (prm->preconditioner && !prm->multigrid && (rc = ensure_factors(h, deta_of(h, prm->dtau)))) return rc;
        if (prm->multigrid && (rc = mg_prepare(h, prm, true))) return rc;
        if (prm->autotune && (rc = autotune_handle(h, prm))) return rc;
        PCF_CUDA_TRY(cudaEventRecord(h->ev[2], h->stream));
        PCF_CUDA_TRY(cudaMemsetAsync(h->x64, 0, sizeof(double) * h->d.n, h->stream));
        // r = b - A 0 = b and its sum of squares
        k_copy_sumsq<<<vec_grid(h->d.n), 256, 0, h->stream>>>(h->b64, h->w64, h->d.n,
                                                               red(h, nullptr, FIN_STORE, h->dot_out));
        h->launches += 1;
        PCF_CUDA_TRY(cudaGetLastError());
        PCF_CUDA_TRY(cudaMemcpyAsync(e->h_norm + q, h->dot_out, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    }
    for (int q = 0; q < n; ++q) PCF_CUDA_TRY(cudaStreamSynchronize(e->m[q]->stream));
    // the iteration graph, captured with every stream idle
    if (!e->exec || !e->key_valid || e->key_ci != ci || e->key_precond != prm->preconditioner ||
        e->key_pc_iters != prm->preconditioner_iterations || e->key_dtau != prm->dtau || e->key_mg != prm->multigrid ||
        e->key_mg_ci != prm->mg_coarse_iterations || e->key_mg_min != prm->mg_min_columns ||
        e->key_mg_dtau != prm->mg_dtau || e->key_maxit != prm->poisson_iterations) {
        if ((rc = ensemble_capture(e, prm, ci))) return rc;
    }
    std::vector<double> bnorm(n), tol(n);
    std::vector<char> active(n, 0);
    int nactive = 0;
    for (int q = 0; q < n; ++q) {
        pcf_handle *h = e->m[q];
        tol[q] = prm->tolerance_is_relative ? prm->tolerance : prm->tolerance / tolref[q];
        bnorm[q] = std::sqrt(e->h_norm[q] / (double)h->d.n);
        res[q].b_norm = bnorm[q];
        if (!std::isfinite(bnorm[q])) {
            res[q].status = PCF_ENONFINITE;
            res[q].errflag = 1;
        } else if (bnorm[q] > 0.0 && 1.0 > tol[q]) {
            active[q] = 1;
            nactive += 1;
        }
        if (!active[q]) {
            // the member's kernels in the graph must return at once
            KrylovScalars idle;
            std::memset(&idle, 0, sizeof(idle));
            idle.done = 1;
            PCF_CUDA_TRY(cudaMemcpyAsync(h->scal32, &idle, sizeof(idle), cudaMemcpyHostToDevice, h->stream));
            continue;
        }
        const LoopCfg c = ensemble_loop_cfg(h, prm);
        const Work<float> w = work32_pi(h);
        k_to_float<<<vec_grid(h->d.n), 256, 0, h->stream>>>(h->w64, w.s, h->d.n, 1.0 / bnorm[q]);
        h->launches += 1;
        PCF_CUDA_TRY(cudaGetLastError());
        if ((rc = run_start<float>(h, w, w.s, tol[q], maxit, c, 0, 1.0, bnorm[q], prm->inner_tolerance,
                                   prm->restart_interval)))
            return rc;
    }
    for (int q = 0; q < n; ++q) {
        PCF_CUDA_TRY(cudaEventRecord(e->join[q], e->m[q]->stream));
        PCF_CUDA_TRY(cudaStreamWaitEvent(e->origin, e->join[q], 0));
    }
    PCF_CUDA_TRY(cudaEventRecord(e->t1, e->origin));
    // the whole iteration as one graph launch (the loop decides on the device
    // when every member has finished); without conditional nodes, one graph
    // launch per batch with the status of batch b read while b + 1 runs
    int launched = 0, inflight = 0, slot = 0;
    bool all_done = nactive == 0;
    if (!all_done && e->loop_exec) {
        PCF_CUDA_TRY(cudaMemsetAsync(e->d_batches, 0, sizeof(int), e->origin));
        PCF_CUDA_TRY(cudaGraphLaunch(e->loop_exec, e->origin));
        int batches = 0;
        PCF_CUDA_TRY(cudaMemcpyAsync(&batches, e->d_batches, sizeof(int), cudaMemcpyDeviceToHost, e->origin));
        PCF_CUDA_TRY(cudaStreamSynchronize(e->origin));
        e->launches += e->graph_launches * batches + batches;  // + the loop's control kernel
        all_done = true;
    }
    while (!all_done) {
        if (launched < maxit) {
            PCF_CUDA_TRY(cudaGraphLaunch(e->exec, e->origin));
            e->launches += e->graph_launches;
            launched += ci;
            for (int q = 0; q < n; ++q)
                if (active[q])
                    PCF_CUDA_TRY(cudaMemcpyAsync(e->h_status + slot * n + q, e->m[q]->scal32, sizeof(KrylovScalars),
                                                 cudaMemcpyDeviceToHost, e->origin));
            PCF_CUDA_TRY(cudaEventRecord(e->slot_ev[slot], e->origin));
            slot ^= 1;
            inflight += 1;
        }
        if (inflight == 0) break;
        if (inflight == 2 || launched >= maxit) {
            const int old = (inflight == 2) ? slot : slot ^ 1;
            PCF_CUDA_TRY(cudaEventSynchronize(e->slot_ev[old]));
            inflight -= 1;
            bool all = true;
            for (int q = 0; q < n; ++q)
                if (active[q] && !e->h_status[old * n + q].done) all = false;
            all_done = all;
            if (launched >= maxit && inflight == 0) break;
        }
    }
    PCF_CUDA_TRY(cudaEventRecord(e->done, e->origin));
    // outcomes; a member whose FP32 iteration broke down is solved again by
    // the single-handle solver (with its restarts after a breakdown)
    for (int q = 0; q < n; ++q) {
        pcf_handle *h = e->m[q];
        PCF_CUDA_TRY(cudaStreamWaitEvent(h->stream, e->done, 0));
        const double *x = h->x64;
        if (active[q]) {
            const LoopCfg c = ensemble_loop_cfg(h, prm);
            const Work<float> w = work32_pi(h);
            float *xe = nullptr;
            RunOut ro;
            if ((rc = run_finish<float>(h, w, c, false, 0, &xe, &ro))) return rc;
            res[q].niter = ro.iters;
            res[q].nrefine = ro.nupdates;
            reliable_bytes(h, ro.nupdates);
            res[q].status = ro.status;
            res[q].residual = res[q].true_residual = ro.nupdates > 0 ? ro.res : 1.0;
            res[q].errflag = ro.converged ? 0 : 1;
            if (!ro.converged && ro.status == PCF_EBREAKDOWN) {
                pcf_result r2;
                std::memset(&r2, 0, sizeof(r2));
                if ((rc = krylov_solve(h, tolref[q], prm, &x, &r2))) return rc;
                r2.niter += res[q].niter;
                r2.nrefine += res[q].nrefine;
                res[q] = r2;
            }
        } else if (res[q].status == PCF_OK) {
            res[q].residual = res[q].true_residual = 0.0;
        }
        PCF_CUDA_TRY(cudaEventRecord(h->ev[3], h->stream));
        if (!res[q].errflag) {
            k_unscale<<<vec_grid(h->d.n), 256, 0, h->stream>>>(x, h->pbar, h->rhobar, 1.0 / dt[q], h->d.nx, h->d.ny,
                                                               h->d.nz, h->dims.nbx, h->dims.nby, h->dims.nbz, h->nxx,
                                                               h->nyy, d_dpip[q], h->dims.nbx, h->dims.nby,
                                                               h->dims.nbz, h->nxx, h->nyy);
            h->launches += 1;
            PCF_CUDA_TRY(cudaGetLastError());
        }
        PCF_CUDA_TRY(cudaEventRecord(h->ev[4], h->stream));
        PCF_CUDA_TRY(cudaEventRecord(e->join[q], h->stream));
        PCF_CUDA_TRY(cudaStreamWaitEvent(e->origin, e->join[q], 0));
    }
    PCF_CUDA_TRY(cudaEventRecord(e->t2, e->origin));
    PCF_CUDA_TRY(cudaEventSynchronize(e->t2));
    const float total = elapsed(e->t0, e->t2), loop = elapsed(e->t1, e->done);
    for (int q = 0; q < n; ++q) {
        pcf_handle *h = e->m[q];
        res[q].ms_upload = elapsed(h->ev[0], h->ev[1]);
        res[q].ms_assemble = elapsed(h->ev[1], h->ev[2]);
        res[q].ms_solve = loop;
        res[q].ms_download = elapsed(h->ev[3], h->ev[4]);
        res[q].ms_total = total;
    }
    return PCF_OK;
}

}  // extern "C"
