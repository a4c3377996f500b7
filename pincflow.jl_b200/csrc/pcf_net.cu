// pcf_net.cu -- the learned preconditioner / warm start (no reference
// counterpart): a per-column MLP fused with full 3x3 horizontal
// convolutions, BF16 weights and activations, FP32 accumulation on the
// tensor cores, trained on the GPU with the kernels in this file (forward,
// backward, Adam).
//
// Per column c of the nx x ny grid, x = the column of a field resampled to
// L = 64 levels and im2col(v)[c] = (v[nbr(c, t)], t = 0..8) its periodic
// 3 x 3 window (tap t = (dj+1)*3 + (di+1) is the neighbour (i+di, j+dj)):
//   a  = relu(C1 im2col(x) + c1)        64      C1: 64 x 576
//   h1 = relu(W1 a + b1)                256
//   h2 = relu(W2 h1 + b2)               256
//   z  = W3 h2 + b3                     64
//   y  = z + C2 im2col(z) + c2          64      C2: 64 x 576
// 172,736 parameters.
//
// Two implementations of the forward pass:
//  * the application (pcf_net_apply_device: warm start, preconditioner
//    stage) is ONE cooperative kernel, k_net_fused: it gathers the input
//    columns into a haloed BF16 array, then for every tile of 16 x 8 columns
//    runs the input convolution and the three dense layers back to back on
//    tcgen05 with the activations in tensor memory and shared memory (TMA
//    brings each 3 x 3 window and each weight K-block into shared memory),
//    writes z, and after a grid-wide barrier runs the output convolution and
//    resamples y back onto the field's levels;
//  * training (pcf_net_train_step, pcf_net_train) keeps every activation for
//    the backward pass: the convolutions become GEMMs over im2col matrices on
//    the general tcgen05 GEMM of pcf_umma.cuh.
// Both round to BF16 at the same points, so they agree to FP32 summation
// order.
#include <cuda.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "pcf_internal.cuh"
#include "pcf_umma.cuh"

namespace pcf {
namespace net {

using bf16 = __nv_bfloat16;

constexpr int L = 64, HID = 256, TAPS = 9, KC = TAPS * L;  // KC: the im2col width, 576
constexpr int OFF_C1 = 0;                    // [L][KC]
constexpr int OFF_c1 = OFF_C1 + L * KC;      // [L]
constexpr int OFF_W1 = OFF_c1 + L;           // [HID][L]
constexpr int OFF_B1 = OFF_W1 + HID * L;     // [HID]
constexpr int OFF_W2 = OFF_B1 + HID;         // [HID][HID]
constexpr int OFF_B2 = OFF_W2 + HID * HID;   // [HID]
constexpr int OFF_W3 = OFF_B2 + HID;         // [L][HID]
constexpr int OFF_B3 = OFF_W3 + L * HID;     // [L]
constexpr int OFF_C2 = OFF_B3 + L;           // [L][KC]
constexpr int OFF_c2 = OFF_C2 + L * KC;      // [L]
constexpr int NPARAM = OFF_c2 + L;           // 172,736
// the BF16 weight copies, one array: C1 | W1 | W2 | W3 | C2
constexpr int WB_C1 = 0, WB_W1 = WB_C1 + L * KC, WB_W2 = WB_W1 + HID * L, WB_W3 = WB_W2 + HID * HID,
              WB_C2 = WB_W3 + L * HID, WB_N = WB_C2 + L * KC;
constexpr int KSPLIT = 32;                   // split-K of the weight-gradient GEMMs
constexpr int RED_CHUNK = 64;                // columns per block of the column reductions

// ------------------------------------------------------------ launchers --

// The dynamic shared-memory attribute is a per-device setting of a kernel, so
// it is recorded per device (up to 64) and kernel instance.
template <int NT>
static int launch_gemm(const umma::GemmArgs &g, int ksplit, cudaStream_t st) {
    static std::atomic<unsigned long long> attr_set{0};
    constexpr int smem = umma::gemm_smem_bytes<NT>();
    int dev = 0;
    PCF_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return PCF_ENODEVICE;
    if (!(attr_set.load() >> dev & 1ull)) {
        const cudaError_t e =
            cudaFuncSetAttribute(umma::k_gemm_bf16<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return pcf_set_cuda_error(e);
        attr_set.fetch_or(1ull << dev);
    }
    const int ksteps = (g.K + 63) / 64;
    if (ksplit > ksteps) ksplit = ksteps;
    if (ksplit < 1) ksplit = 1;
    const dim3 grid((unsigned)((g.M + 127) / 128), 1, (unsigned)ksplit);
    umma::k_gemm_bf16<NT><<<grid, 128, smem, st>>>(g);
    PCF_CUDA_TRY(cudaGetLastError());
    return PCF_OK;
}

// D = A B^T with the tile width chosen from N.
static int gemm(const umma::GemmArgs &g, int ksplit, cudaStream_t st) {
    if (g.N <= 64) return launch_gemm<64>(g, ksplit, st);
    if (g.N <= 128) return launch_gemm<128>(g, ksplit, st);
    if (g.N <= 256) return launch_gemm<256>(g, ksplit, st);
    return PCF_ERANGE;
}

static umma::GemmArgs gargs(int M, int N, int K, const bf16 *A, long long a_rs, long long a_ks, const bf16 *B,
                            long long b_rs, long long b_ks, int *err) {
    umma::GemmArgs g{};
    g.M = M;
    g.N = N;
    g.K = K;
    g.A = A;
    g.a_rs = a_rs;
    g.a_ks = a_ks;
    g.B = B;
    g.b_rs = b_rs;
    g.b_ks = b_ks;
    g.error = err;
    return g;
}

// ------------------------------------------------------------------ state --

struct Net {
    int device;
    cudaStream_t stream;
    long long cap;  // column capacity of an application
    float *param, *grad, *m, *v;
    bf16 *wb;       // BF16 weight copies (WB_* offsets)
    // the fused application: haloed input columns and z, grid barrier
    bf16 *xh, *zh;
    long long hcap;  // haloed columns xh / zh hold
    unsigned *bar;
    CUtensorMap wmap[5];  // C1, W1, W2, W3, C2 (K-block boxes)
    CUtensorMap xmap, zmap;
    int map_nx, map_ny;
    // training activations and gradients (allocated on first use, tcap columns)
    long long tcap;
    bf16 *x0, *xi, *a, *h1, *h2, *zb, *zi, *dyb, *dzb, *dg2b, *dg1b, *dgab;
    float *y, *t, *dyf, *dzf, *dh, *dzi, *part;
    double *red, *scal;   // loss partial sums; [0] numerator, [1] sum t^2, [2] loss
    int *err;
    int step;
    int no_bias;  // biases held at zero: N is then positively homogeneous, N(a x) = a N(x) for a > 0
};

// ------------------------------------------------------- column transfers --

// level position of output level l when resampling n_in levels to n_out
__device__ __forceinline__ void interp_pos(int l, int n_in, int n_out, int &k0, int &k1, float &f) {
    if (n_in == n_out) {
        k0 = k1 = l;
        f = 0.f;
        return;
    }
    float pos = ((float)l + 0.5f) * (float)n_in / (float)n_out - 0.5f;
    pos = fminf(fmaxf(pos, 0.f), (float)(n_in - 1));
    k0 = (int)floorf(pos);
    k1 = min(k0 + 1, n_in - 1);
    f = pos - (float)k0;
}

// field (nz levels, x fastest) -> X[c][l] (L levels), times scale
template <typename TIn, typename TOut>
__global__ void k_gather(const TIn *__restrict__ field, long long plane, int nz, float scale, TOut *__restrict__ X) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= plane * L) return;
    const int l = (int)(idx / plane);
    const long long c = idx % plane;
    int k0, k1;
    float f;
    interp_pos(l, nz, L, k0, k1, f);
    const float v = (1.f - f) * (float)field[k0 * plane + c] + f * (float)field[k1 * plane + c];
    X[c * L + l] = (TOut)(scale * v);
}

__device__ __forceinline__ long long nbr(long long c, int nx, int ny, int tap) {
    const int di = tap % 3 - 1, dj = tap / 3 - 1;
    const int i = (int)(c % nx), j = (int)(c / nx);
    const int ii = (i + di + nx) % nx, jj = (j + dj + ny) % ny;
    return (long long)jj * nx + ii;
}

// im2col of a [C][L] BF16 array: out[c][t*L + l] = H[nbr(c, t)][l], one thread per 16 bytes
__global__ void k_im2col(const bf16 *__restrict__ H, long long C, int nx, int ny, bf16 *__restrict__ out) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= C * TAPS * (L / 8)) return;
    const int q = (int)(idx % (L / 8));
    const int t = (int)((idx / (L / 8)) % TAPS);
    const long long c = idx / (TAPS * (L / 8));
    const uint4 v = *reinterpret_cast<const uint4 *>(H + nbr(c, nx, ny, t) * L + q * 8);
    *reinterpret_cast<uint4 *>(out + c * KC + t * L + q * 8) = v;
}

// The adjoint of im2col plus the residual path of the output convolution:
// dz[c][l] = dy[c][l] + sum_t D[nbr(c, 8 - t)][t*L + l] (FP32 and BF16)
__global__ void k_col2im(const float *__restrict__ D, const float *__restrict__ dy, long long C, int nx, int ny,
                         float *__restrict__ dz, bf16 *__restrict__ dzb) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= C * L) return;
    const long long c = idx / L;
    const int l = (int)(idx % L);
    float acc = dy[idx];
#pragma unroll
    for (int t = 0; t < TAPS; ++t) acc += D[nbr(c, nx, ny, TAPS - 1 - t) * KC + t * L + l];
    dz[idx] = acc;
    dzb[idx] = __float2bfloat16(acc);
}

// y += z (the output convolution's residual path)
__global__ void k_add_bf16(float *__restrict__ y, const bf16 *__restrict__ z, long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) y[i] += __bfloat162float(z[i]);
}

// ------------------------------------------------------------- reductions --

// sum over the first dimension: out[j] = sum_b in[b * n + j] (fixed order)
__global__ void k_sum_rows(const float *__restrict__ in, int rows, int n, float *__restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    float acc = 0.f;
    for (int b = 0; b < rows; ++b) acc += in[(long long)b * n + j];
    out[j] = acc;
}

// the same for split-K partials of a transposed gradient: in[b][k][o]
// (rows x K x O) summed into out[o][k]
__global__ void k_sum_rows_t(const float *__restrict__ in, int rows, int K, int O, float *__restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;  // j = o * K + k
    if (j >= K * O) return;
    const int o = j / K, k = j % K;
    float acc = 0.f;
    for (int b = 0; b < rows; ++b) acc += in[((long long)b * K + k) * O + o];
    out[j] = acc;
}

// residual-weighted loss sum (Y - T)^2 / sum T^2: per-block partial sums
__global__ void k_loss_part(const float *__restrict__ Y, const float *__restrict__ T, long long n,
                            double *__restrict__ part) {
    __shared__ double s1[256], s2[256];
    double a = 0, b = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double d = (double)Y[i] - (double)T[i];
        a += d * d;
        b += (double)T[i] * (double)T[i];
    }
    s1[threadIdx.x] = a;
    s2[threadIdx.x] = b;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s1[threadIdx.x] += s1[threadIdx.x + o];
            s2[threadIdx.x] += s2[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = s1[0];
        part[2 * blockIdx.x + 1] = s2[0];
    }
}

// final loss; also stored to log[slot] (log nullable)
__global__ void k_loss_final(const double *__restrict__ part, int nb, double *__restrict__ scal, double *log,
                             int slot) {
    double a = 0, b = 0;
    for (int i = 0; i < nb; ++i) {
        a += part[2 * i];
        b += part[2 * i + 1];
    }
    scal[0] = a;
    scal[1] = b;
    scal[2] = b > 0 ? a / b : a;
    if (log) log[slot] = scal[2];
}

// dL/dY = 2 (Y - T) / sum T^2 (FP32 and BF16)
__global__ void k_dy(const float *__restrict__ Y, const float *__restrict__ T, long long n,
                     const double *__restrict__ scal, float *__restrict__ dyf, bf16 *__restrict__ dyb) {
    const double w = scal[1] > 0 ? 2.0 / scal[1] : 2.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float g = (float)(w * ((double)Y[i] - (double)T[i]));
        dyf[i] = g;
        dyb[i] = __float2bfloat16(g);
    }
}

// column sums of a [C][F] FP32 array, per block of RED_CHUNK columns
__global__ void k_colsum_part(const float *__restrict__ a, long long C, int F, float *__restrict__ part) {
    const int f = threadIdx.x;
    const long long c0 = (long long)blockIdx.x * RED_CHUNK;
    float acc = 0.f;
    for (long long c = c0; c < c0 + RED_CHUNK && c < C; ++c) acc += a[c * F + f];
    part[(long long)blockIdx.x * F + f] = acc;
}

// backward through a ReLU: g = dh * (h > 0) as BF16, with the per-block
// column sums of g (the bias gradient) for RED_CHUNK columns
__global__ void k_relu_bwd(const float *__restrict__ dh, const bf16 *__restrict__ h, long long C, int F,
                           bf16 *__restrict__ g, float *__restrict__ part) {
    const int f = threadIdx.x;
    const long long c0 = (long long)blockIdx.x * RED_CHUNK;
    float acc = 0.f;
    for (long long c = c0; c < c0 + RED_CHUNK && c < C; ++c) {
        const float v = __bfloat162float(h[c * F + f]) > 0.f ? dh[c * F + f] : 0.f;
        g[c * F + f] = __float2bfloat16(v);
        acc += v;
    }
    part[(long long)blockIdx.x * F + f] = acc;
}

// ------------------------------------------------------------------ Adam --

__host__ __device__ constexpr bool is_bias(int i) {
    return (i >= OFF_c1 && i < OFF_c1 + L) || (i >= OFF_B1 && i < OFF_B1 + HID) ||
           (i >= OFF_B2 && i < OFF_B2 + HID) || (i >= OFF_B3 && i < OFF_B3 + L) || (i >= OFF_c2 && i < OFF_c2 + L);
}

// index of parameter i in the BF16 weight copies, -1 for a bias
__device__ __forceinline__ int wb_index(int i) {
    if (i < OFF_c1) return WB_C1 + (i - OFF_C1);
    if (i >= OFF_W1 && i < OFF_B1) return WB_W1 + (i - OFF_W1);
    if (i >= OFF_W2 && i < OFF_B2) return WB_W2 + (i - OFF_W2);
    if (i >= OFF_W3 && i < OFF_B3) return WB_W3 + (i - OFF_W3);
    if (i >= OFF_C2 && i < OFF_c2) return WB_C2 + (i - OFF_C2);
    return -1;
}

// Adam (FP32 master weights), then the BF16 copy of the updated weight
__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2,
                       bf16 *__restrict__ wb, int no_bias) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (no_bias && is_bias(i)) return;  // held at zero
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    const int w = wb_index(i);
    if (w >= 0) wb[w] = __float2bfloat16(pi);
}

__global__ void k_params_to_bf16(const float *__restrict__ p, bf16 *__restrict__ wb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NPARAM) return;
    const int w = wb_index(i);
    if (w >= 0) wb[w] = __float2bfloat16(p[i]);
}

// ================================================= the fused application --
//
// One cooperative launch of 192-thread CTAs, one per SM (its shared memory
// holds one), each owning all 512 TMEM columns:
//   phase 0  gather: xh[(yh)(nx+2) + xh][l] = BF16(scale_in * column
//            (xh-1, yh-1) of the input, resampled to L levels), periodic
//            halo of one column included;
//   barrier;
//   phase 1  per tile of 16 x 8 columns (M = 128 rows): 9 K-steps of the
//            input convolution (A = the TMA box of xh shifted by the tap, B =
//            the tap's 64 x 64 block of C1), the dense layers W1 (1 step, A =
//            the activations in shared memory), W2 (4 steps), W3 (4 steps);
//            z (BF16) goes to zh, periodic images included;
//   barrier;
//   phase 2  per tile: 9 K-steps of the output convolution over zh, then
//            y = z + C2 im2col(z) + c2, resampled to the nz levels of the
//            output: out = beta * out + scale_out * y.
// Warp roles: warp 4 (one thread) streams every TMA box of the CTA's K-steps
// through a four-stage ring, as far ahead as the ring allows (the weights
// and the windows of xh do not depend on the activations); warp 5 (one
// thread) issues the tcgen05.mma of each K-step once its stage has landed,
// frees the stage with tcgen05.commit, and signals each finished layer;
// warps 0-3 (one TMEM lane = one tile row per thread) run the epilogues --
// bias, ReLU, BF16 into the shared operand of the next layer, or z / y to
// global memory -- and signal that the accumulator and operand are ready.
// Shared-memory operand layout (TMA boxes land in it directly): K-major
// with the 128-byte swizzle, one 64-value K-block per operand block: row r
// is the 128 bytes at r * 128, its 16-byte chunk c at ((c ^ (r % 8)) * 16),
// 8-row groups 1024 B apart (SBO); blocks are 1024-byte aligned.  A TMA box
// row is then 128 bytes, and a K-step of 16 values advances the descriptor's
// start address by 32 bytes.
// Every wait is bounded (2 s of %globaltimer); a role that gives up stops,
// the others give up on their next wait, and all leave after the grid
// barriers (bounded too) with the error flag set.

constexpr int F_TX = 16, F_TY = 8, F_ROWS = F_TX * F_TY;  // tile = 128 rows
constexpr int F_THREADS = 192;                             // warps 0-3 epilogue, 4 copies, 5 MMAs
constexpr int F_STAGES = 4;
constexpr int F_SZA = F_ROWS * L * 2;                      // 16 KB: an A K-block (128 x 64)
constexpr int F_SZS = HID * L * 2;                         // 32 KB stage: a B K-block (256 x 64), or
                                                           // A (16 KB) + B (64 x 64, 8 KB) of a window
constexpr int F_OFF_S = 0;                                 // F_STAGES stages
constexpr int F_OFF_ACT = F_OFF_S + F_STAGES * F_SZS;      // a: one A K-block
constexpr int F_OFF_H = F_OFF_ACT + F_SZA;                 // h1 / h2: 4 A K-blocks; y in phase 2
constexpr int F_NBIAS = L + HID + HID + L + L;             // c1 | b1 | b2 | b3 | c2
constexpr int F_OFF_BIAS = F_OFF_H + 4 * F_SZA;
constexpr int F_OFF_GTAB = F_OFF_BIAS + 4 * F_NBIAS;       // resampling nz -> L: L entries
constexpr int F_OFF_STAB = F_OFF_GTAB + 8 * L;             // resampling L -> nz: F_STAB entries
constexpr int F_STAB = 1536;                               // levels beyond it are computed on the fly
constexpr int F_OFF_BAR = F_OFF_STAB + 8 * F_STAB;
constexpr int F_NBAR = 2 * F_STAGES + 2;                   // full[], empty[], acc_full, epi_done
constexpr int F_SMEM = F_OFF_BAR + 8 * F_NBAR + 16;        // 228,704 bytes
constexpr int F_SMEM_ALLOC = F_SMEM + 1024;                // the layout starts at the next 1024-byte boundary
constexpr int F_TMEM_COLS = 512;
constexpr int F_COL64 = 0, F_COL256 = 256;                 // accumulators: N = 64 and N = 256

// The layers of a tile, in order: phase 1 runs C1, W1, W2, W3; phase 2 C2.
enum FLayer { F_C1 = 0, F_W1 = 1, F_W2 = 2, F_W3 = 3, F_C2 = 4 };
__host__ __device__ constexpr int f_steps(int l) { return l == F_W1 ? 1 : (l == F_W2 || l == F_W3) ? HID / 64 : TAPS; }
__host__ __device__ constexpr int f_n(int l) { return (l == F_W1 || l == F_W2) ? HID : L; }
__host__ __device__ constexpr bool f_conv(int l) { return l == F_C1 || l == F_C2; }

struct FusedArgs {
    const void *in;
    void *out;
    int nx, ny, nz;
    float scale_in, scale_out, beta;
    const float *param;  // FP32 parameters (the biases)
    bf16 *xh, *zh;
    unsigned *bar;       // grid barrier counter, zero at launch
    int *err;
};

// Shared-memory matrix descriptor, K-major, 128-byte swizzle (layout type 2,
// bits [61,64)); SBO = 1024 B between 8-row groups; LBO unused for this
// layout (set to 16 B).
__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr) {
    return umma::smem_desc(saddr, 16, 1024) | ((uint64_t)2 << 61);
}

__device__ __forceinline__ void tma2(uint32_t dst, const CUtensorMap *map, int c0, int c1, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tma3(uint32_t dst, const CUtensorMap *map, int c0, int c1, int c2, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
        "%4}], [%5];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void arrive_expect(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mma_f16(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
        "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

// 32 consecutive FP32 accumulator columns of this thread's TMEM lane (row)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&f)[32]) {
    uint32_t v[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 32; ++q) f[q] = __uint_as_float(v[q]);
}

// the two source levels and the weight of the second, for resampling level l
struct Interp {
    unsigned short k0, k1;
    float f;
};
__device__ __forceinline__ Interp make_interp(int l, int n_in, int n_out) {
    int k0, k1;
    float f;
    interp_pos(l, n_in, n_out, k0, k1, f);
    return Interp{(unsigned short)k0, (unsigned short)k1, f};
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    const __nv_bfloat162 p = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&p);
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d)
                 : "memory");
}

// out[0..3] = (beta ? beta * out : 0) + v, four consecutive values
__device__ __forceinline__ void store4(float *o, float v0, float v1, float v2, float v3, float beta) {
    float4 r = make_float4(v0, v1, v2, v3);
    if (beta != 0.f) {
        const float4 p = *reinterpret_cast<const float4 *>(o);
        r = make_float4(beta * p.x + v0, beta * p.y + v1, beta * p.z + v2, beta * p.w + v3);
    }
    *reinterpret_cast<float4 *>(o) = r;
}
__device__ __forceinline__ void store4(double *o, float v0, float v1, float v2, float v3, float beta) {
    double2 r0 = make_double2(v0, v1), r1 = make_double2(v2, v3);
    if (beta != 0.f) {
        const double2 p0 = reinterpret_cast<const double2 *>(o)[0], p1 = reinterpret_cast<const double2 *>(o)[1];
        r0 = make_double2((double)((float)beta * (float)p0.x + v0), (double)((float)beta * (float)p0.y + v1));
        r1 = make_double2((double)((float)beta * (float)p1.x + v2), (double)((float)beta * (float)p1.y + v3));
    }
    reinterpret_cast<double2 *>(o)[0] = r0;
    reinterpret_cast<double2 *>(o)[1] = r1;
}

// barrier among the 128 epilogue threads only (named barrier 1)
__device__ __forceinline__ void epilogue_sync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

// Grid-wide barrier of a cooperative launch: one arrival per CTA on a
// counter that starts at zero, wait until it reaches `target`; every thread's
// generic writes before it become visible to TMA reads after it.  Bounded.
// Returns false for every thread if the barrier gave up or any thread
// arrived with ok = false.
__device__ bool grid_barrier(unsigned *bar, unsigned target, bool ok) {
    __syncwarp();  // a warp whose lane 0 ran a role alone reconverges first
    asm volatile("fence.proxy.async.global;" ::: "memory");
    __syncthreads();
    int fail = ok ? 0 : 1;
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(bar, 1u);
        uint64_t t0, t1;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
        for (;;) {
            unsigned v;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(bar) : "memory");
            if (v >= target) break;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
            if (t1 - t0 > 2000000000ull) {
                fail = 1;
                break;
            }
            __nanosleep(64);
        }
    }
    const bool passed = __syncthreads_or(fail) == 0;
    asm volatile("fence.proxy.async.global;" ::: "memory");
    return passed;
}

// accumulator columns [tcol, tcol + ncols) + bias, ReLU, as BF16 into the
// shared K-blocks at dst (K-block b at dst + b * F_SZA); thread = row
__device__ __forceinline__ void epi_to_smem(uint32_t tmem, uint32_t tcol, const float *bias, int ncols, bool relu,
                                            uint32_t dst) {
    const int warp = threadIdx.x >> 5, r = threadIdx.x;
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16) + tcol;
#pragma unroll 1
    for (int c0 = 0; c0 < ncols; c0 += 32) {
        float f[32];
        tmem_ld32(lane_base + (uint32_t)c0, f);
#pragma unroll
        for (int q = 0; q < 32; ++q) {
            f[q] += bias[c0 + q];
            if (relu) f[q] = fmaxf(f[q], 0.f);
        }
        const uint32_t row = dst + (uint32_t)(c0 >> 6) * F_SZA + (uint32_t)r * 128;
        const int q8 = (c0 & 63) >> 3;
#pragma unroll
        for (int h = 0; h < 4; ++h)
            st_shared_v4(row + (uint32_t)(((q8 + h) ^ (r & 7)) * 16), pack_bf16x2(f[8 * h], f[8 * h + 1]),
                         pack_bf16x2(f[8 * h + 2], f[8 * h + 3]), pack_bf16x2(f[8 * h + 4], f[8 * h + 5]),
                         pack_bf16x2(f[8 * h + 6], f[8 * h + 7]));
    }
}

// Producer: the TMA boxes of one layer's K-steps into the ring.  A window
// step's stage holds A at its start and B 16 KB in; a dense step's holds B.
struct Producer {
    uint32_t ss, full[F_STAGES], empty[F_STAGES];
    unsigned g;  // K-steps issued so far
    __device__ bool layer(int l, const CUtensorMap *amap, const CUtensorMap *bmap, int x0, int y0) {
        const bool conv = f_conv(l);
        const uint32_t bytes = (uint32_t)f_n(l) * L * 2 + (conv ? (uint32_t)F_SZA : 0u);
        for (int i = 0; i < f_steps(l); ++i, ++g) {
            const int s = (int)(g % F_STAGES);
            const unsigned use = g / F_STAGES;
            // the stage's previous use must have been consumed by its MMAs
            if (use > 0 && !mbar_wait(empty[s], (use - 1u) & 1u)) return false;
            arrive_expect(full[s], bytes);
            const uint32_t st = ss + s * F_SZS;
            if (conv) tma3(st, amap, 0, x0 + i % 3, y0 + i / 3, full[s]);
            tma2(st + (conv ? F_SZA : 0), bmap, 64 * i, 0, full[s]);
        }
        return true;
    }
};

// MMA issuer: one layer's K-steps into its accumulator, then the layer's signal.
struct Issuer {
    uint32_t ss, full[F_STAGES], empty[F_STAGES], acc_full, epi_done, tmem;
    unsigned g, nepi;
    bool first;
    __device__ bool layer(int l, uint32_t abase) {
        // the previous layer's epilogue has read its accumulator and written this layer's operand
        if (!first) {
            if (!mbar_wait(epi_done, nepi & 1u)) return false;
            ++nepi;
        }
        first = false;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int nn = f_n(l);
        const bool conv = f_conv(l);
        const uint32_t idesc = umma::instr_desc(128, nn);
        const uint32_t tcol = nn == HID ? F_COL256 : F_COL64;
        for (int i = 0; i < f_steps(l); ++i, ++g) {
            const int s = (int)(g % F_STAGES);
            if (!mbar_wait(full[s], (g / F_STAGES) & 1u)) return false;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t st = ss + s * F_SZS;
            const uint32_t abuf = conv ? st : abase + (uint32_t)i * F_SZA;
            const uint32_t bbuf = conv ? st + F_SZA : st;
#pragma unroll
            for (int j = 0; j < 4; ++j)  // K = 16 per instruction: 32 bytes along the swizzled rows
                mma_f16(tmem + tcol, desc_sw128(abuf + 32 * j), desc_sw128(bbuf + 32 * j), idesc,
                        (i > 0 || j > 0) ? 1u : 0u);
            mma_commit(empty[s]);
        }
        mma_commit(acc_full);
        return true;
    }
};

template <typename T>
__global__ void __launch_bounds__(F_THREADS, 1)
    k_net_fused(const __grid_constant__ CUtensorMap mx, const __grid_constant__ CUtensorMap mz,
                const __grid_constant__ CUtensorMap mc1, const __grid_constant__ CUtensorMap mw1,
                const __grid_constant__ CUtensorMap mw2, const __grid_constant__ CUtensorMap mw3,
                const __grid_constant__ CUtensorMap mc2, const FusedArgs a) {
    extern __shared__ __align__(1024) uint8_t sm_raw[];
    // the swizzled operand blocks must start on 1024-byte boundaries
    uint8_t *sm = sm_raw + ((1024u - (smem_u32(sm_raw) & 1023u)) & 1023u);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + F_OFF_BAR);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + F_NBAR);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(F_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int q = 0; q < F_NBAR; ++q)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bars + q)),
                         "r"(q == F_NBAR - 1 ? 128 : 1));  // epi_done: one arrival per epilogue thread
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tslot;
    uint32_t full[F_STAGES], empty[F_STAGES];
    for (int q = 0; q < F_STAGES; ++q) {
        full[q] = smem_u32(bars + q);
        empty[q] = smem_u32(bars + F_STAGES + q);
    }
    const uint32_t acc_full = smem_u32(bars + 2 * F_STAGES), epi_done = smem_u32(bars + 2 * F_STAGES + 1);
    const uint32_t ss = smem_u32(sm + F_OFF_S);
    const uint32_t s_act = smem_u32(sm + F_OFF_ACT), s_h = smem_u32(sm + F_OFF_H);

    const int nx = a.nx, ny = a.ny, nz = a.nz, nxh = nx + 2, nyh = ny + 2;
    const long long plane = (long long)nx * ny;
    const int ntx = (nx + F_TX - 1) / F_TX, nty = (ny + F_TY - 1) / F_TY, ntiles = ntx * nty;
    bool ok = true;
    // the biases and the level-resampling tables in shared memory
    float *bias = reinterpret_cast<float *>(sm + F_OFF_BIAS);
    Interp *gtab = reinterpret_cast<Interp *>(sm + F_OFF_GTAB), *stab = reinterpret_cast<Interp *>(sm + F_OFF_STAB);
    for (int i = tid; i < F_NBIAS; i += blockDim.x)
        bias[i] = i < L ? a.param[OFF_c1 + i]
                : i < L + HID ? a.param[OFF_B1 + i - L]
                : i < L + 2 * HID ? a.param[OFF_B2 + i - L - HID]
                : i < 2 * L + 2 * HID ? a.param[OFF_B3 + i - L - 2 * HID] : a.param[OFF_c2 + i - 2 * L - 2 * HID];
    for (int i = tid; i < L; i += blockDim.x) gtab[i] = make_interp(i, nz, L);
    for (int i = tid; i < min(nz, F_STAB); i += blockDim.x) stab[i] = make_interp(i, L, nz);
    __syncthreads();
    const float *b_c1 = bias, *b_b1 = bias + L, *b_b2 = bias + L + HID, *b_b3 = bias + L + 2 * HID,
                *b_c2 = bias + 2 * L + 2 * HID;

    // ---- phase 0: the haloed input columns, 8 levels (16 bytes) per thread
    // (four units per thread and pass, every load issued before the first is
    // used: one CTA per SM needs many loads in flight; 32-bit indices, the
    // haloed column count is below 2^28)
    {
        const T *in = static_cast<const T *>(a.in);
        const unsigned cols = (unsigned)nxh * (unsigned)nyh, units = cols * (L / 8);
        const unsigned stride = gridDim.x * blockDim.x;
        for (unsigned u0 = blockIdx.x * blockDim.x + tid; u0 < units; u0 += 4 * stride) {
            float x0[4][8], x1[4][8];
            unsigned dst[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const unsigned u = min(u0 + r * stride, units - 1);
                const unsigned col = u % cols, q = u / cols;
                const unsigned xh = col % (unsigned)nxh, yh = col / (unsigned)nxh;
                const int x = xh == 0 ? nx - 1 : ((int)xh > nx ? 0 : (int)xh - 1);
                const int y = yh == 0 ? ny - 1 : ((int)yh > ny ? 0 : (int)yh - 1);
                const long long c = (long long)y * nx + x;
                dst[r] = col * L + q * 8;
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    const Interp w = gtab[q * 8 + e];
                    x0[r][e] = (float)in[w.k0 * plane + c];
                    x1[r][e] = (float)in[w.k1 * plane + c];
                }
            }
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                if (u0 + r * stride >= units) continue;
                const unsigned q = (dst[r] % L) / 8;
                float v[8];
#pragma unroll
                for (int e = 0; e < 8; ++e) {
                    const float f = gtab[q * 8 + e].f;
                    v[e] = a.scale_in * ((1.f - f) * x0[r][e] + f * x1[r][e]);
                }
                *reinterpret_cast<uint4 *>(a.xh + dst[r]) =
                    make_uint4(pack_bf16x2(v[0], v[1]), pack_bf16x2(v[2], v[3]), pack_bf16x2(v[4], v[5]),
                               pack_bf16x2(v[6], v[7]));
            }
        }
    }
    ok = grid_barrier(a.bar, gridDim.x, ok);

    Producer P;
    Issuer I;
    P.ss = I.ss = ss;
    for (int q = 0; q < F_STAGES; ++q) {
        P.full[q] = I.full[q] = full[q];
        P.empty[q] = I.empty[q] = empty[q];
    }
    P.g = I.g = 0;
    I.acc_full = acc_full;
    I.epi_done = epi_done;
    I.tmem = tmem;
    I.nepi = 0;
    I.first = true;
    unsigned nacc = 0;  // epilogue: accumulators waited for
    // epilogue: wait for a layer's accumulator (a warp-uniform outcome: the
    // TMEM loads that follow are warp-collective)
    auto wait_acc = [&]() -> bool {
        const bool r = __all_sync(0xffffffffu, mbar_wait(acc_full, nacc & 1u));
        ++nacc;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        return r;
    };
    // epilogue: accumulator read, operand written (visible to the tensor core)
    auto epi_signal = [&]() {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        arrive(epi_done);
    };

    // ---- phase 1: input convolution and the dense layers, z to zh
    if (ok) {
        if (warp == 4) {
            if (lane == 0)
                for (int tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x) {
                    const int x0 = (tile % ntx) * F_TX, y0 = (tile / ntx) * F_TY;
                    // the haloed window of tap t starts at (x0 + t % 3, y0 + t / 3)
                    ok = P.layer(F_C1, &mx, &mc1, x0, y0) && P.layer(F_W1, nullptr, &mw1, 0, 0) &&
                         P.layer(F_W2, nullptr, &mw2, 0, 0) && P.layer(F_W3, nullptr, &mw3, 0, 0);
                }
        } else if (warp == 5) {
            if (lane == 0)
                for (int tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x)
                    ok = I.layer(F_C1, 0) && I.layer(F_W1, s_act) && I.layer(F_W2, s_h) && I.layer(F_W3, s_h);
        } else {
            for (int tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x) {
                const int x0 = (tile % ntx) * F_TX, y0 = (tile / ntx) * F_TY;
                if (!(ok = wait_acc())) break;
                epi_to_smem(tmem, F_COL64, b_c1, L, true, s_act);
                epi_signal();
                if (!(ok = wait_acc())) break;
                epi_to_smem(tmem, F_COL256, b_b1, HID, true, s_h);
                epi_signal();
                if (!(ok = wait_acc())) break;
                epi_to_smem(tmem, F_COL256, b_b2, HID, true, s_h);
                epi_signal();
                if (!(ok = wait_acc())) break;
                // z = acc + b3 as BF16, to the interior row and its periodic images in zh
                const int x = x0 + (tid % F_TX), y = y0 + (tid / F_TX);
                uint32_t pk[32];
                const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16) + F_COL64;
#pragma unroll
                for (int c0 = 0; c0 < L; c0 += 32) {
                    float f[32];
                    tmem_ld32(lane_base + (uint32_t)c0, f);
#pragma unroll
                    for (int q = 0; q < 16; ++q)
                        pk[c0 / 2 + q] = pack_bf16x2(f[2 * q] + b_b3[c0 + 2 * q], f[2 * q + 1] + b_b3[c0 + 2 * q + 1]);
                }
                epi_signal();
                if (x < nx && y < ny) {
                    const int xs[3] = {x + 1, x == nx - 1 ? 0 : -1, x == 0 ? nx + 1 : -1};
                    const int ys[3] = {y + 1, y == ny - 1 ? 0 : -1, y == 0 ? ny + 1 : -1};
                    for (int p = 0; p < 3; ++p)
                        for (int o = 0; o < 3; ++o) {
                            if (ys[p] < 0 || xs[o] < 0) continue;
                            uint4 *dst = reinterpret_cast<uint4 *>(a.zh + ((long long)ys[p] * nxh + xs[o]) * L);
#pragma unroll
                            for (int q = 0; q < 8; ++q)
                                dst[q] = make_uint4(pk[4 * q], pk[4 * q + 1], pk[4 * q + 2], pk[4 * q + 3]);
                        }
                }
            }
        }
    }
    ok = grid_barrier(a.bar, 2u * gridDim.x, ok);

    // ---- phase 2: output convolution, residual, resampling to nz levels
    if (ok) {
        if (warp == 4) {
            if (lane == 0)
                for (int tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x) {
                    const int x0 = (tile % ntx) * F_TX, y0 = (tile / ntx) * F_TY;
                    ok = P.layer(F_C2, &mz, &mc2, x0, y0);
                }
        } else if (warp == 5) {
            if (lane == 0)
                for (int tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x) ok = I.layer(F_C2, 0);
        } else {
            float *ysm = reinterpret_cast<float *>(sm + F_OFF_H);  // y of the tile, [L][128]
            T *out = static_cast<T *>(a.out);
            // vector stores need rows of a multiple of 4 values and an aligned field
            const bool vec4 = nx % 4 == 0 && (reinterpret_cast<uintptr_t>(out) & (4 * sizeof(T) - 1)) == 0;
            for (int tile = blockIdx.x; ok && tile < ntiles; tile += gridDim.x) {
                const int x0 = (tile % ntx) * F_TX, y0 = (tile / ntx) * F_TY;
                const int x = x0 + (tid % F_TX), y = y0 + (tid / F_TX);
                const bool inside = x < nx && y < ny;
                if (!(ok = wait_acc())) break;
                float acc[L];
                const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16) + F_COL64;
#pragma unroll
                for (int c0 = 0; c0 < L; c0 += 32) {
                    float f[32];
                    tmem_ld32(lane_base + (uint32_t)c0, f);
#pragma unroll
                    for (int q = 0; q < 32; ++q) acc[c0 + q] = f[q];
                }
                epi_signal();  // the accumulator is free for the next tile's MMAs
                const uint4 *zr = reinterpret_cast<const uint4 *>(a.zh + ((long long)(y + 1) * nxh + (x + 1)) * L);
#pragma unroll
                for (int q = 0; q < L / 8; ++q) {
                    const uint4 zq = inside ? zr[q] : make_uint4(0, 0, 0, 0);
                    const __nv_bfloat16 *zb = reinterpret_cast<const __nv_bfloat16 *>(&zq);
#pragma unroll
                    for (int e = 0; e < 8; ++e)
                        ysm[(q * 8 + e) * F_ROWS + tid] =
                            acc[q * 8 + e] + b_c2[q * 8 + e] + __bfloat162float(zb[e]);
                }
                epilogue_sync();
                if (vec4 && x0 + F_TX <= nx) {
                    // four consecutive x per thread and level (16-byte rows of y in
                    // shared memory, vector stores): thread = (level phase, tile row, x group)
                    const int lo = tid >> 5, yr = (tid >> 2) & 7, xg = tid & 3;
                    if (y0 + yr < ny) {
                        const long long c = (long long)(y0 + yr) * nx + x0 + 4 * xg;
                        const int row = yr * F_TX + 4 * xg;
                        for (int k = lo; k < nz; k += 4) {
                            const Interp w = k < F_STAB ? stab[k] : make_interp(k, L, nz);
                            const float4 p0 = *reinterpret_cast<const float4 *>(ysm + w.k0 * F_ROWS + row);
                            const float4 p1 = *reinterpret_cast<const float4 *>(ysm + w.k1 * F_ROWS + row);
                            const float g0 = a.scale_out * (1.f - w.f), g1 = a.scale_out * w.f;
                            store4(out + (long long)k * plane + c, g0 * p0.x + g1 * p1.x, g0 * p0.y + g1 * p1.y,
                                   g0 * p0.z + g1 * p1.z, g0 * p0.w + g1 * p1.w, a.beta);
                        }
                    }
                } else if (inside) {
                    const long long c = (long long)y * nx + x;
                    for (int k = 0; k < nz; ++k) {
                        const Interp w = k < F_STAB ? stab[k] : make_interp(k, L, nz);
                        const float v =
                            a.scale_out * ((1.f - w.f) * ysm[w.k0 * F_ROWS + tid] + w.f * ysm[w.k1 * F_ROWS + tid]);
                        T *o = out + (long long)k * plane + c;
                        *o = a.beta == 0.f ? (T)v : (T)((float)a.beta * (float)*o + v);
                    }
                }
                epilogue_sync();  // before the next tile overwrites y
            }
        }
    }
    __syncwarp();
    if (__syncthreads_or(!ok) && tid == 0 && a.err) atomicExch(a.err, 1);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(F_TMEM_COLS));
}

// ---------------------------------------------------------- tensor maps --

using EncodeFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                              const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeFn encoder() {
    static EncodeFn fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return static_cast<EncodeFn>(nullptr);
        }
        return reinterpret_cast<EncodeFn>(f);
    }();
    return fn;
}

// A weight matrix W[N][K] (BF16, row-major), boxes of 64 x N: one K-block of
// 64 values of every row, 128-byte swizzled.
static bool weight_map(CUtensorMap *m, const bf16 *w, int N, int K) {
    EncodeFn enc = encoder();
    if (!enc) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)N};
    const cuuint64_t strides[1] = {2ull * K};
    const cuuint32_t box[2] = {64, (cuuint32_t)N};
    const cuuint32_t estr[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16 *>(w), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Haloed columns H[(yh)(nx+2) + xh][L] seen as (l, xh, yh), boxes of 64 x 16
// x 8: the 128 rows of a tile (x fastest) of one window, 128-byte swizzled.
static bool column_map(CUtensorMap *m, const bf16 *h, int nx, int ny) {
    EncodeFn enc = encoder();
    if (!enc) return false;
    const cuuint64_t dims[3] = {L, (cuuint64_t)(nx + 2), (cuuint64_t)(ny + 2)};
    const cuuint64_t strides[2] = {2ull * L, 2ull * L * (nx + 2)};
    const cuuint32_t box[3] = {L, F_TX, F_TY};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<bf16 *>(h), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// CTAs of the cooperative launch on the net's device: one per SM (each
// holds all 512 TMEM columns); 0 if the device refuses the shared memory.
template <typename T>
static int fused_grid(Net &n) {
    static std::atomic<unsigned long long> attr_set{0};
    if (!(attr_set.load() >> n.device & 1ull)) {
        PCF_CUDA_TRY(cudaFuncSetAttribute(k_net_fused<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, F_SMEM_ALLOC));
        attr_set.fetch_or(1ull << n.device);
    }
    int per_sm = 0, sms = 0;
    PCF_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_net_fused<T>, F_THREADS, F_SMEM_ALLOC));
    PCF_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, n.device));
    if (per_sm < 1) return 0;
    return sms;
}

template <typename T>
static int apply_fused(Net &n, const void *in, int nx, int ny, int nz, float si, float so, float beta, void *out,
                       cudaStream_t st) {
    if ((long long)(nx + 2) * (ny + 2) > n.hcap || (long long)(nx + 2) * (ny + 2) >= (1ll << 28)) return PCF_ERANGE;
    if (n.map_nx != nx || n.map_ny != ny) {
        if (!column_map(&n.xmap, n.xh, nx, ny) || !column_map(&n.zmap, n.zh, nx, ny)) return PCF_ECUDA;
        n.map_nx = nx;
        n.map_ny = ny;
    }
    const int cap = fused_grid<T>(n);
    if (cap < 1) return PCF_ECUDA;
    const int ntiles = ((nx + F_TX - 1) / F_TX) * ((ny + F_TY - 1) / F_TY);
    const int grid = std::max(1, std::min(cap, ntiles));
    PCF_CUDA_TRY(cudaMemsetAsync(n.bar, 0, sizeof(unsigned), st));
    FusedArgs a{};
    a.in = in;
    a.out = out;
    a.nx = nx;
    a.ny = ny;
    a.nz = nz;
    a.scale_in = si;
    a.scale_out = so;
    a.beta = beta;
    a.param = n.param;
    a.xh = n.xh;
    a.zh = n.zh;
    a.bar = n.bar;
    a.err = n.err;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(F_THREADS);
    cfg.dynamicSmemBytes = F_SMEM_ALLOC;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    PCF_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_net_fused<T>, n.xmap, n.zmap, n.wmap[0], n.wmap[1], n.wmap[2], n.wmap[3],
                                    n.wmap[4], a));
    return PCF_OK;
}

// ============================================== training (unfused) path --

static int alloc_training(Net &n, long long C) {
    if (C <= n.tcap) return PCF_OK;
    void *ptrs[] = {n.x0, n.xi, n.a, n.h1, n.h2, n.zb, n.zi, n.dyb, n.dzb, n.dg2b, n.dg1b, n.dgab,
                    n.y, n.t, n.dyf, n.dzf, n.dh, n.dzi, n.part};
    PCF_CUDA_TRY(cudaStreamSynchronize(n.stream));
    for (void *q : ptrs)
        if (q) cudaFree(q);
    n.tcap = 0;
    auto A = [&](void **q, size_t b) -> int {
        *q = nullptr;
        const cudaError_t e = cudaMalloc(q, b);
        return e == cudaSuccess ? PCF_OK : pcf_set_cuda_error(e);
    };
    const size_t f4 = sizeof(float), b2 = sizeof(bf16);
    const long long nchunk = (C + RED_CHUNK - 1) / RED_CHUNK;
    const size_t part = std::max<size_t>({(size_t)KSPLIT * KC * L, (size_t)KSPLIT * HID * HID,
                                          (size_t)nchunk * HID});
    int rc;
    if ((rc = A((void **)&n.x0, C * L * b2)) || (rc = A((void **)&n.xi, C * KC * b2)) ||
        (rc = A((void **)&n.a, C * L * b2)) || (rc = A((void **)&n.h1, C * HID * b2)) ||
        (rc = A((void **)&n.h2, C * HID * b2)) || (rc = A((void **)&n.zb, C * L * b2)) ||
        (rc = A((void **)&n.zi, C * KC * b2)) || (rc = A((void **)&n.dyb, C * L * b2)) ||
        (rc = A((void **)&n.dzb, C * L * b2)) || (rc = A((void **)&n.dg2b, C * HID * b2)) ||
        (rc = A((void **)&n.dg1b, C * HID * b2)) || (rc = A((void **)&n.dgab, C * L * b2)) ||
        (rc = A((void **)&n.y, C * L * f4)) || (rc = A((void **)&n.t, C * L * f4)) ||
        (rc = A((void **)&n.dyf, C * L * f4)) || (rc = A((void **)&n.dzf, C * L * f4)) ||
        (rc = A((void **)&n.dh, C * HID * f4)) || (rc = A((void **)&n.dzi, C * KC * f4)) ||
        (rc = A((void **)&n.part, part * f4)))
        return rc;
    n.tcap = C;
    return PCF_OK;
}

static unsigned blocks(long long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// Forward on the columns already gathered into n.x0 (C columns), keeping
// every activation: a, h1, h2, z (BF16), the im2col matrices, y (FP32).
static int forward_train(Net &n, long long C, int nx, int ny) {
    cudaStream_t st = n.stream;
    int rc;
    const int M = (int)C;
    k_im2col<<<blocks(C * TAPS * (L / 8)), 256, 0, st>>>(n.x0, C, nx, ny, n.xi);
    umma::GemmArgs g = gargs(M, L, KC, n.xi, KC, 1, n.wb + WB_C1, KC, 1, n.err);
    g.bias = n.param + OFF_c1;
    g.relu = 1;
    g.outB = n.a;
    if ((rc = gemm(g, 1, st))) return rc;
    g = gargs(M, HID, L, n.a, L, 1, n.wb + WB_W1, L, 1, n.err);
    g.bias = n.param + OFF_B1;
    g.relu = 1;
    g.outB = n.h1;
    if ((rc = gemm(g, 1, st))) return rc;
    g = gargs(M, HID, HID, n.h1, HID, 1, n.wb + WB_W2, HID, 1, n.err);
    g.bias = n.param + OFF_B2;
    g.relu = 1;
    g.outB = n.h2;
    if ((rc = gemm(g, 1, st))) return rc;
    g = gargs(M, L, HID, n.h2, HID, 1, n.wb + WB_W3, HID, 1, n.err);
    g.bias = n.param + OFF_B3;
    g.outB = n.zb;
    if ((rc = gemm(g, 1, st))) return rc;
    k_im2col<<<blocks(C * TAPS * (L / 8)), 256, 0, st>>>(n.zb, C, nx, ny, n.zi);
    g = gargs(M, L, KC, n.zi, KC, 1, n.wb + WB_C2, KC, 1, n.err);
    g.bias = n.param + OFF_c2;
    g.outF = n.y;
    if ((rc = gemm(g, 1, st))) return rc;
    k_add_bf16<<<blocks(C * L), 256, 0, st>>>(n.y, n.zb, C * L);
    PCF_CUDA_TRY(cudaGetLastError());
    return PCF_OK;
}

// weight gradient D[o][k] = sum_c G[c][o] X[c][k] (G: C x O BF16, X: C x K
// BF16), split-K over the columns, summed into grad (row-major O x K)
static int weight_grad(Net &n, const bf16 *G, int O, const bf16 *X, int K, long long C, float *grad) {
    cudaStream_t st = n.stream;
    const int used = std::min<int>(KSPLIT, (int)((C + 63) / 64));
    int rc;
    if (K <= 256) {
        umma::GemmArgs g = gargs(O, K, (int)C, G, 1, O, X, 1, K, n.err);
        g.outF = n.part;
        if ((rc = gemm(g, KSPLIT, st))) return rc;
        k_sum_rows<<<blocks((long long)O * K), 256, 0, st>>>(n.part, used, O * K, grad);
    } else {  // K = 576 (a convolution): D^T[k][o] with M = K, N = O, transposed in the sum
        umma::GemmArgs g = gargs(K, O, (int)C, X, 1, K, G, 1, O, n.err);
        g.outF = n.part;
        if ((rc = gemm(g, KSPLIT, st))) return rc;
        k_sum_rows_t<<<blocks((long long)O * K), 256, 0, st>>>(n.part, used, K, O, grad);
    }
    PCF_CUDA_TRY(cudaGetLastError());
    return PCF_OK;
}

// bias gradient: column sums of a C x F FP32 array
static void bias_grad(Net &n, const float *a, long long C, int F, float *grad) {
    const unsigned nchunk = (unsigned)((C + RED_CHUNK - 1) / RED_CHUNK);
    k_colsum_part<<<nchunk, F, 0, n.stream>>>(a, C, F, n.part);
    k_sum_rows<<<1, F, 0, n.stream>>>(n.part, (int)nchunk, F, grad);
}

// Loss and gradients (into n.grad) for targets already gathered into n.t.
static int backward(Net &n, long long C, int nx, int ny, double *log, int slot) {
    cudaStream_t st = n.stream;
    int rc;
    const int M = (int)C;
    const unsigned nchunk = (unsigned)((C + RED_CHUNK - 1) / RED_CHUNK);
    k_loss_part<<<256, 256, 0, st>>>(n.y, n.t, C * L, n.red);
    k_loss_final<<<1, 1, 0, st>>>(n.red, 256, n.scal, log, slot);
    k_dy<<<1024, 256, 0, st>>>(n.y, n.t, C * L, n.scal, n.dyf, n.dyb);
    // output convolution: c2, C2, then dz = dy + col2im(dy C2)
    bias_grad(n, n.dyf, C, L, n.grad + OFF_c2);
    if ((rc = weight_grad(n, n.dyb, L, n.zi, KC, C, n.grad + OFF_C2))) return rc;
    for (int nb = 0; nb < 3; ++nb) {  // dzi = dy C2 in three column blocks of 192
        umma::GemmArgs g = gargs(M, 192, L, n.dyb, L, 1, n.wb + WB_C2 + nb * 192, 1, KC, n.err);
        g.outF = n.dzi + nb * 192;
        g.ldo = KC;
        if ((rc = gemm(g, 1, st))) return rc;
    }
    k_col2im<<<blocks(C * L), 256, 0, st>>>(n.dzi, n.dyf, C, nx, ny, n.dzf, n.dzb);
    // W3, b3; dh2 = dz W3
    bias_grad(n, n.dzf, C, L, n.grad + OFF_B3);
    if ((rc = weight_grad(n, n.dzb, L, n.h2, HID, C, n.grad + OFF_W3))) return rc;
    umma::GemmArgs g = gargs(M, HID, L, n.dzb, L, 1, n.wb + WB_W3, 1, HID, n.err);
    g.outF = n.dh;
    if ((rc = gemm(g, 1, st))) return rc;
    k_relu_bwd<<<nchunk, HID, 0, st>>>(n.dh, n.h2, C, HID, n.dg2b, n.part);
    k_sum_rows<<<1, HID, 0, st>>>(n.part, (int)nchunk, HID, n.grad + OFF_B2);
    // W2; dh1 = dg2 W2
    if ((rc = weight_grad(n, n.dg2b, HID, n.h1, HID, C, n.grad + OFF_W2))) return rc;
    g = gargs(M, HID, HID, n.dg2b, HID, 1, n.wb + WB_W2, 1, HID, n.err);
    g.outF = n.dh;
    if ((rc = gemm(g, 1, st))) return rc;
    k_relu_bwd<<<nchunk, HID, 0, st>>>(n.dh, n.h1, C, HID, n.dg1b, n.part);
    k_sum_rows<<<1, HID, 0, st>>>(n.part, (int)nchunk, HID, n.grad + OFF_B1);
    // W1; da = dg1 W1
    if ((rc = weight_grad(n, n.dg1b, HID, n.a, L, C, n.grad + OFF_W1))) return rc;
    g = gargs(M, L, HID, n.dg1b, HID, 1, n.wb + WB_W1, 1, L, n.err);
    g.outF = n.dh;
    if ((rc = gemm(g, 1, st))) return rc;
    k_relu_bwd<<<nchunk, L, 0, st>>>(n.dh, n.a, C, L, n.dgab, n.part);
    k_sum_rows<<<1, L, 0, st>>>(n.part, (int)nchunk, L, n.grad + OFF_c1);
    // input convolution: C1
    if ((rc = weight_grad(n, n.dgab, L, n.xi, KC, C, n.grad + OFF_C1))) return rc;
    PCF_CUDA_TRY(cudaGetLastError());
    return PCF_OK;
}

static int check_err(Net &n) {
    int e = 0;
    PCF_CUDA_TRY(cudaMemcpyAsync(&e, n.err, sizeof(int), cudaMemcpyDeviceToHost, n.stream));
    PCF_CUDA_TRY(cudaStreamSynchronize(n.stream));
    return e ? PCF_ECUDA : PCF_OK;
}

// gather b (the input) and x (the target) of one sample, forward, backward,
// and (lr > 0) an Adam step; the loss goes to log[slot] (nullable)
static int train_one(Net &n, const float *b, const float *x, int nx, int ny, int nz, double lr, double *log,
                     int slot) {
    const long long C = (long long)nx * ny;
    int rc;
    if ((rc = alloc_training(n, C))) return rc;
    cudaStream_t st = n.stream;
    k_gather<float, bf16><<<blocks(C * L), 256, 0, st>>>(b, C, nz, 1.0f, n.x0);
    k_gather<float, float><<<blocks(C * L), 256, 0, st>>>(x, C, nz, 1.0f, n.t);
    PCF_CUDA_TRY(cudaGetLastError());
    if ((rc = forward_train(n, C, nx, ny))) return rc;
    if ((rc = backward(n, C, nx, ny, log, slot))) return rc;
    if (lr > 0) {
        n.step += 1;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - std::pow(b1, (float)n.step), c2 = 1.f - std::pow(b2, (float)n.step);
        k_adam<<<blocks(NPARAM), 256, 0, st>>>(n.param, n.grad, n.m, n.v, NPARAM, (float)lr, b1, b2, 1e-8f, c1, c2,
                                               n.wb, n.no_bias);
        PCF_CUDA_TRY(cudaGetLastError());
    }
    return PCF_OK;
}

}  // namespace net
}  // namespace pcf

struct pcf_net {
    pcf::net::Net n;
};

using namespace pcf::net;

extern "C" {

// Test entry point for the tensor-core GEMM: D[M][N] = sum_k A(m,k) B(n,k)
// with BF16 inputs given as uint16 bit patterns (A(m,k) = A[m*a_rs + k*a_ks],
// B(n,k) = B[n*b_rs + k*b_ks]), FP32 output; ksplit > 1 returns the sum of the
// split-K partials.  Host arrays; device 0.
int pcf_gemm_bf16(const unsigned short *A, long long a_len, long long a_rs, long long a_ks, const unsigned short *B,
                  long long b_len, long long b_rs, long long b_ks, int M, int N, int K, int ksplit, float *D) {
    if (!A || !B || !D || M < 1 || N < 1 || N > 256 || K < 1 || a_len < 1 || b_len < 1) return PCF_EINVAL;
    if (a_rs < 0 || a_ks < 0 || b_rs < 0 || b_ks < 0) return PCF_EINVAL;
    // every element the kernel reads must lie inside the given arrays
    if ((M - 1) * a_rs + (K - 1) * a_ks >= a_len || (N - 1) * b_rs + (K - 1) * b_ks >= b_len) return PCF_ERANGE;
    if (!(a_ks == 1 || a_rs == 1) || !(b_ks == 1 || b_rs == 1)) return PCF_EINVAL;
    bf16 *dA = nullptr, *dB = nullptr;
    float *dD = nullptr;
    int *derr = nullptr;
    const int ks = std::max(1, ksplit);
    int rc = PCF_OK;
    cudaError_t e;
    if ((e = cudaMalloc(&dA, a_len * 2)) != cudaSuccess || (e = cudaMalloc(&dB, b_len * 2)) != cudaSuccess ||
        (e = cudaMalloc(&dD, sizeof(float) * (size_t)M * N * ks)) != cudaSuccess ||
        (e = cudaMalloc(&derr, sizeof(int))) != cudaSuccess) {
        rc = pcf_set_cuda_error(e);
    }
    if (!rc) {
        cudaMemcpy(dA, A, a_len * 2, cudaMemcpyHostToDevice);
        cudaMemcpy(dB, B, b_len * 2, cudaMemcpyHostToDevice);
        cudaMemset(dD, 0, sizeof(float) * (size_t)M * N * ks);
        cudaMemset(derr, 0, sizeof(int));
        pcf::umma::GemmArgs g{};
        g.M = M;
        g.N = N;
        g.K = K;
        g.A = dA;
        g.a_rs = a_rs;
        g.a_ks = a_ks;
        g.B = dB;
        g.b_rs = b_rs;
        g.b_ks = b_ks;
        g.outF = dD;
        g.error = derr;
        rc = gemm(g, ks, 0);
        if (!rc) {
            e = cudaDeviceSynchronize();
            if (e != cudaSuccess) rc = pcf_set_cuda_error(e);
        }
        if (!rc) {
            int herr = 0;
            cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost);
            if (herr) rc = PCF_ECUDA;
        }
        if (!rc) {
            std::vector<float> part((size_t)M * N * ks);
            cudaMemcpy(part.data(), dD, sizeof(float) * part.size(), cudaMemcpyDeviceToHost);
            const int used = ks;
            for (size_t i = 0; i < (size_t)M * N; ++i) {
                float acc = 0;
                for (int z = 0; z < used; ++z) acc += part[(size_t)z * M * N + i];
                D[i] = acc;
            }
        }
    }
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dD);
    cudaFree(derr);
    return rc;
}

}  // extern "C"

// ===================================================================== C ABI

namespace {

// Deterministic initialisation: He-uniform C1, W1, W2; zero W3, C2 and
// biases, so that the untrained network outputs zero (loss 1 against any
// target) and training starts from "no correction".
void init_params(std::vector<float> &p, unsigned seed) {
    uint64_t s = 0x9E3779B97F4A7C15ull ^ (uint64_t)seed;
    auto uni = [&]() {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        return (double)(s >> 11) * (1.0 / 9007199254740992.0);
    };
    p.assign(NPARAM, 0.0f);
    auto fill = [&](int off, int n, int fan_in) {
        const double a = std::sqrt(6.0 / fan_in);
        for (int i = 0; i < n; ++i) p[off + i] = (float)((2 * uni() - 1) * a);
    };
    fill(OFF_C1, L * KC, KC);
    fill(OFF_W1, HID * L, L);
    fill(OFF_W2, HID * HID, HID);
}

int net_upload_params(Net &n, const float *host) {
    PCF_CUDA_TRY(cudaMemcpyAsync(n.param, host, NPARAM * sizeof(float), cudaMemcpyHostToDevice, n.stream));
    k_params_to_bf16<<<(NPARAM + 255) / 256, 256, 0, n.stream>>>(n.param, n.wb);
    PCF_CUDA_TRY(cudaGetLastError());
    PCF_CUDA_TRY(cudaStreamSynchronize(n.stream));
    return PCF_OK;
}

int net_alloc(Net &n, long long cap) {
    auto A = [&](void **q, size_t b) -> int {
        const cudaError_t e = cudaMalloc(q, b);
        return e == cudaSuccess ? PCF_OK : pcf_set_cuda_error(e);
    };
    const size_t f4 = sizeof(float);
    // a grid of at most cap columns has at most 3 cap + 6 haloed columns (ny = 1)
    n.hcap = 3 * cap + 6;
    int rc;
    if ((rc = A((void **)&n.param, NPARAM * f4)) || (rc = A((void **)&n.grad, NPARAM * f4)) ||
        (rc = A((void **)&n.m, NPARAM * f4)) || (rc = A((void **)&n.v, NPARAM * f4)) ||
        (rc = A((void **)&n.wb, WB_N * sizeof(bf16))) || (rc = A((void **)&n.xh, n.hcap * L * sizeof(bf16))) ||
        (rc = A((void **)&n.zh, n.hcap * L * sizeof(bf16))) || (rc = A((void **)&n.bar, sizeof(unsigned))) ||
        (rc = A((void **)&n.red, 512 * sizeof(double))) || (rc = A((void **)&n.scal, 4 * sizeof(double))) ||
        (rc = A((void **)&n.err, sizeof(int))))
        return rc;
    if (!weight_map(&n.wmap[0], n.wb + WB_C1, L, KC) || !weight_map(&n.wmap[1], n.wb + WB_W1, HID, L) ||
        !weight_map(&n.wmap[2], n.wb + WB_W2, HID, HID) || !weight_map(&n.wmap[3], n.wb + WB_W3, L, HID) ||
        !weight_map(&n.wmap[4], n.wb + WB_C2, L, KC))
        return PCF_ECUDA;
    n.map_nx = n.map_ny = -1;
    return PCF_OK;
}

}  // namespace

extern "C" {

int pcf_net_num_params(void) { return NPARAM; }

int pcf_net_create(pcf_net **out, int device, long long max_columns, unsigned seed) {
    if (!out || max_columns < 1) return PCF_EINVAL;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return PCF_ENODEVICE;
    PCF_CUDA_TRY(cudaSetDevice(device));
    pcf_net *w = new pcf_net;
    std::memset(&w->n, 0, sizeof(w->n));
    w->n.device = device;
    w->n.cap = max_columns;
    int rc = PCF_OK;
    if (cudaStreamCreateWithFlags(&w->n.stream, cudaStreamNonBlocking) != cudaSuccess) rc = PCF_ECUDA;
    if (!rc) rc = net_alloc(w->n, max_columns);
    std::vector<float> p;
    init_params(p, seed);
    if (!rc) rc = net_upload_params(w->n, p.data());
    if (!rc) {
        cudaMemsetAsync(w->n.m, 0, NPARAM * sizeof(float), w->n.stream);
        cudaMemsetAsync(w->n.v, 0, NPARAM * sizeof(float), w->n.stream);
        cudaMemsetAsync(w->n.grad, 0, NPARAM * sizeof(float), w->n.stream);
        cudaMemsetAsync(w->n.err, 0, sizeof(int), w->n.stream);
        if (cudaStreamSynchronize(w->n.stream) != cudaSuccess) rc = PCF_ECUDA;
    }
    if (rc) {
        pcf_net_destroy(w);
        return rc;
    }
    *out = w;
    return PCF_OK;
}

int pcf_net_destroy(pcf_net *w) {
    if (!w) return PCF_OK;
    Net &n = w->n;
    cudaSetDevice(n.device);
    if (n.stream) cudaStreamSynchronize(n.stream);
    void *ptrs[] = {n.param, n.grad, n.m,   n.v,   n.wb,  n.xh,   n.zh,   n.bar,  n.red, n.scal, n.err,
                    n.x0,    n.xi,   n.a,   n.h1,  n.h2,  n.zb,   n.zi,   n.dyb,  n.dzb, n.dg2b, n.dg1b,
                    n.dgab,  n.y,    n.t,   n.dyf, n.dzf, n.dh,   n.dzi,  n.part};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    if (n.stream) cudaStreamDestroy(n.stream);
    delete w;
    return PCF_OK;
}

int pcf_net_get_params(pcf_net *w, float *host) {
    if (!w || !host) return PCF_EINVAL;
    PCF_CUDA_TRY(cudaSetDevice(w->n.device));
    PCF_CUDA_TRY(cudaStreamSynchronize(w->n.stream));
    PCF_CUDA_TRY(cudaMemcpy(host, w->n.param, NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
    return PCF_OK;
}

int pcf_net_set_params(pcf_net *w, const float *host) {
    if (!w || !host) return PCF_EINVAL;
    PCF_CUDA_TRY(cudaSetDevice(w->n.device));
    w->n.step = 0;
    cudaMemsetAsync(w->n.m, 0, NPARAM * sizeof(float), w->n.stream);
    cudaMemsetAsync(w->n.v, 0, NPARAM * sizeof(float), w->n.stream);
    return net_upload_params(w->n, host);
}

// Network output for a device field: out = beta * out + scale_out * N(scale_in * in),
// by the fused kernel.  in / out: nz x ny x nx (x fastest), device memory;
// double or float by `fp64`.
int pcf_net_apply_device(pcf_net *w, const void *in, int nx, int ny, int nz, double scale_in, double scale_out,
                         double beta, void *out, int fp64, void *stream) {
    if (!w || !in || !out || nx < 1 || ny < 1 || nz < 1) return PCF_EINVAL;
    Net &n = w->n;
    if ((long long)nx * ny > n.cap || nz > 65535) return PCF_ERANGE;
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : n.stream;
    return fp64 ? apply_fused<double>(n, in, nx, ny, nz, (float)scale_in, (float)scale_out, (float)beta, out, st)
                : apply_fused<float>(n, in, nx, ny, nz, (float)scale_in, (float)scale_out, (float)beta, out, st);
}

int pcf_net_set_bias_free(pcf_net *w, int on) {
    if (!w) return PCF_EINVAL;
    Net &n = w->n;
    PCF_CUDA_TRY(cudaSetDevice(n.device));
    n.no_bias = on ? 1 : 0;
    if (on) {
        const int offs[5] = {OFF_c1, OFF_B1, OFF_B2, OFF_B3, OFF_c2}, lens[5] = {L, HID, HID, L, L};
        for (int q = 0; q < 5; ++q)
            for (float *a : {n.param, n.m, n.v})
                PCF_CUDA_TRY(cudaMemsetAsync(a + offs[q], 0, sizeof(float) * lens[q], n.stream));
        PCF_CUDA_TRY(cudaStreamSynchronize(n.stream));
    }
    return PCF_OK;
}

// Host-array forward (tests): out = N(in), both nz x ny x nx doubles.
int pcf_net_forward(pcf_net *w, const double *in, int nx, int ny, int nz, double *out) {
    if (!w || !in || !out || nx < 1 || ny < 1 || nz < 1) return PCF_EINVAL;
    PCF_CUDA_TRY(cudaSetDevice(w->n.device));
    const size_t bytes = sizeof(double) * (size_t)nx * ny * nz;
    double *d = nullptr;
    PCF_CUDA_TRY(cudaMalloc(&d, 2 * bytes));
    int rc = PCF_OK;
    if (cudaMemcpy(d, in, bytes, cudaMemcpyHostToDevice) != cudaSuccess) rc = PCF_ECUDA;
    if (!rc) rc = pcf_net_apply_device(w, d, nx, ny, nz, 1.0, 1.0, 0.0, d + (size_t)nx * ny * nz, 1, nullptr);
    if (!rc && cudaStreamSynchronize(w->n.stream) != cudaSuccess) rc = PCF_ECUDA;
    if (!rc) rc = check_err(w->n);
    if (!rc && cudaMemcpy(out, d + (size_t)nx * ny * nz, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) rc = PCF_ECUDA;
    cudaFree(d);
    return rc;
}

// One training step on one sample (device fields b and x, nz x ny x nx FP32,
// already normalised): residual-weighted loss sum (N(b) - x)^2 / sum x^2 on the
// 64-level columns, gradients, and (lr > 0) an Adam step.  *loss receives the
// loss before the step; grad (nullable, host, NPARAM floats) the gradients.
int pcf_net_train_step(pcf_net *w, const float *b, const float *x, int nx, int ny, int nz, double lr,
                       double *loss, float *grad) {
    if (!w || !b || !x || nx < 1 || ny < 1 || nz < 1) return PCF_EINVAL;
    Net &n = w->n;
    PCF_CUDA_TRY(cudaSetDevice(n.device));
    int rc = train_one(n, b, x, nx, ny, nz, lr, nullptr, 0);
    if (rc) return rc;
    double s[3];
    PCF_CUDA_TRY(cudaMemcpyAsync(s, n.scal, sizeof(s), cudaMemcpyDeviceToHost, n.stream));
    if (grad) PCF_CUDA_TRY(cudaMemcpyAsync(grad, n.grad, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, n.stream));
    PCF_CUDA_TRY(cudaStreamSynchronize(n.stream));
    if ((rc = check_err(n))) return rc;
    if (loss) *loss = s[2];
    return PCF_OK;
}

// Adam over a data set of `count` samples given as host arrays (each nz x ny
// x nx FP32, normalised), uploaded once to device memory held for the call:
// `epochs` passes, each in an order drawn from `seed`; losses (nullable,
// count * epochs doubles) receives the loss of every step.
int pcf_net_train(pcf_net *w, const float *b, const float *x, int count, int nx, int ny, int nz, int epochs,
                  double lr, unsigned seed, double *losses) {
    if (!w || !b || !x || count < 1 || nx < 1 || ny < 1 || nz < 1 || epochs < 1 || !(lr > 0)) return PCF_EINVAL;
    Net &n = w->n;
    PCF_CUDA_TRY(cudaSetDevice(n.device));
    const size_t per = (size_t)nx * ny * nz, bytes = per * sizeof(float) * (size_t)count;
    float *db = nullptr, *dx = nullptr;
    double *dl = nullptr;
    const long long steps = (long long)count * epochs;
    int rc = PCF_OK;
    if (cudaMalloc(&db, bytes) != cudaSuccess || cudaMalloc(&dx, bytes) != cudaSuccess ||
        cudaMalloc(&dl, steps * sizeof(double)) != cudaSuccess)
        rc = PCF_ENOMEM;
    if (!rc && (cudaMemcpyAsync(db, b, bytes, cudaMemcpyHostToDevice, n.stream) != cudaSuccess ||
                cudaMemcpyAsync(dx, x, bytes, cudaMemcpyHostToDevice, n.stream) != cudaSuccess))
        rc = PCF_ECUDA;
    std::vector<int> order(count);
    uint64_t s = 0x2545F4914F6CDD1Dull ^ ((uint64_t)seed << 1);
    long long k = 0;
    for (int ep = 0; !rc && ep < epochs; ++ep) {
        for (int i = 0; i < count; ++i) order[i] = i;
        for (int i = count - 1; i > 0; --i) {  // Fisher-Yates with a xorshift generator
            s ^= s << 13;
            s ^= s >> 7;
            s ^= s << 17;
            std::swap(order[i], order[(int)(s % (uint64_t)(i + 1))]);
        }
        for (int i = 0; !rc && i < count; ++i, ++k)
            rc = train_one(n, db + per * order[i], dx + per * order[i], nx, ny, nz, lr, dl, (int)k);
    }
    if (!rc && losses &&
        cudaMemcpyAsync(losses, dl, steps * sizeof(double), cudaMemcpyDeviceToHost, n.stream) != cudaSuccess)
        rc = PCF_ECUDA;
    if (!rc && cudaStreamSynchronize(n.stream) != cudaSuccess) rc = PCF_ECUDA;
    if (!rc) rc = check_err(n);
    cudaStreamSynchronize(n.stream);
    cudaFree(db);
    cudaFree(dx);
    cudaFree(dl);
    return rc;
}

// Host-array variant for the gradient check: loss and gradients, no update.
int pcf_net_gradients(pcf_net *w, const double *b, const double *x, int nx, int ny, int nz, double *loss,
                      float *grad) {
    if (!w || !b || !x || !grad) return PCF_EINVAL;
    PCF_CUDA_TRY(cudaSetDevice(w->n.device));
    const size_t cnt = (size_t)nx * ny * nz;
    std::vector<float> hb(b, b + cnt), hx(x, x + cnt);
    float *d = nullptr;
    PCF_CUDA_TRY(cudaMalloc(&d, 2 * cnt * sizeof(float)));
    int rc = PCF_OK;
    if (cudaMemcpy(d, hb.data(), cnt * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d + cnt, hx.data(), cnt * 4, cudaMemcpyHostToDevice) != cudaSuccess)
        rc = PCF_ECUDA;
    if (!rc) rc = pcf_net_train_step(w, d, d + cnt, nx, ny, nz, 0.0, loss, grad);
    cudaFree(d);
    return rc;
}

// Weights file: "PCFNET02", int32 NPARAM, int32 Adam step, then NPARAM FP32 values.
int pcf_net_save(pcf_net *w, const char *path) {
    if (!w || !path) return PCF_EINVAL;
    std::vector<float> p(NPARAM);
    int rc = pcf_net_get_params(w, p.data());
    if (rc) return rc;
    FILE *f = std::fopen(path, "wb");
    if (!f) return PCF_EINVAL;
    const int hdr[2] = {NPARAM, w->n.step};
    const bool ok = std::fwrite("PCFNET02", 1, 8, f) == 8 && std::fwrite(hdr, sizeof(int), 2, f) == 2 &&
                    std::fwrite(p.data(), sizeof(float), p.size(), f) == p.size();
    std::fclose(f);
    return ok ? PCF_OK : PCF_EINVAL;
}

int pcf_net_load(pcf_net *w, const char *path) {
    if (!w || !path) return PCF_EINVAL;
    FILE *f = std::fopen(path, "rb");
    if (!f) return PCF_EINVAL;
    char magic[8];
    int hdr[2];
    std::vector<float> p(NPARAM);
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "PCFNET02", 8) == 0 &&
              std::fread(hdr, sizeof(int), 2, f) == 2 && hdr[0] == NPARAM &&
              std::fread(p.data(), sizeof(float), p.size(), f) == p.size();
    std::fclose(f);
    if (!ok) return PCF_EINVAL;
    return pcf_net_set_params(w, p.data());
}

}  // extern "C"

unsigned long long pcf_bounds_take_net() { return pcf_bounds_take_local(); }
