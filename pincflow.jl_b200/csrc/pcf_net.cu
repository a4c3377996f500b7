// pcf_net.cu -- the learned preconditioner / warm start: a per-column MLP
// (64 -> 256 -> 256 -> 64) interleaved with depthwise 3x3 horizontal
// convolutions, BF16 weights and activations, FP32 accumulation, trained on
// the GPU with the kernels in this file (forward, backward, Adam).  The dense
// layers run on the tensor cores through pcf_umma.cuh.
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

// ------------------------------------------------------------------ model --
//
// Per column c of the nx x ny grid (input: the column of a field resampled to
// L = 64 levels, scaled):
//   h1  = relu(W1 x + b1)                 (256)
//   h1c = h1 + dwconv3x3(h1; K1)          depthwise, periodic in x and y
//   h2  = relu(W2 h1c + b2)               (256)
//   h2c = h2 + dwconv3x3(h2; K2)
//   y   = W3 h2c + b3                     (64, resampled back to nz levels)
// Activations are row-major [column][feature]; BF16 where they feed a GEMM.
constexpr int L = 64, HID = 256, TAPS = 9;
constexpr int OFF_W1 = 0;                    // [HID][L]
constexpr int OFF_B1 = OFF_W1 + HID * L;     // [HID]
constexpr int OFF_K1 = OFF_B1 + HID;         // [HID][9], tap = (dj+1)*3 + (di+1)
constexpr int OFF_W2 = OFF_K1 + HID * TAPS;  // [HID][HID]
constexpr int OFF_B2 = OFF_W2 + HID * HID;
constexpr int OFF_K2 = OFF_B2 + HID;
constexpr int OFF_W3 = OFF_K2 + HID * TAPS;  // [L][HID]
constexpr int OFF_B3 = OFF_W3 + L * HID;     // [L]
constexpr int NPARAM = OFF_B3 + L;           // 103,488
constexpr int KSPLIT = 32;                   // split-K of the weight-gradient GEMMs
constexpr int RED_CHUNK = 64;                // columns per block of the column reductions

struct Net {
    int device;
    cudaStream_t stream;
    long long cap;  // column capacity
    float *param, *grad, *m, *v;
    bf16 *w1b, *w2b, *w3b;
    bf16 *x0, *h1, *h1c, *h2, *h2c, *dyb, *dz2, *dz1;
    float *y, *t, *dyf, *dh2c, *dh1c, *part, *red;
    double *scal;  // [0] loss numerator, [1] sum T^2, [2] loss
    int *err;
    int step;
    int no_bias;  // biases held at zero: N is then positively homogeneous, N(a x) = a N(x) for a > 0
};

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

// Y[c][l] (L levels) -> field (nz levels): out = beta * out + scale * interp(Y)
template <typename TOut>
__global__ void k_scatter(const float *__restrict__ Y, long long plane, int nz, float scale, float beta,
                          TOut *__restrict__ out) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= plane * nz) return;
    const int k = (int)(idx / plane);
    const long long c = idx % plane;
    int l0, l1;
    float f;
    interp_pos(k, L, nz, l0, l1, f);
    const float v = scale * ((1.f - f) * Y[c * L + l0] + f * Y[c * L + l1]);
    out[idx] = beta == 0.f ? (TOut)v : (TOut)((float)beta * (float)out[idx] + v);
}

__device__ __forceinline__ long long nbr(long long c, int nx, int ny, int tap) {
    const int di = tap % 3 - 1, dj = tap / 3 - 1;
    const int i = (int)(c % nx), j = (int)(c / nx);
    const int ii = (i + di + nx) % nx, jj = (j + dj + ny) % ny;
    return (long long)jj * nx + ii;
}

// out = in + depthwise 3x3 conv(in), one thread per (column, channel)
__global__ void k_dwconv(const bf16 *__restrict__ in, const float *__restrict__ Kw, int nx, int ny,
                         bf16 *__restrict__ out) {
    const long long c = blockIdx.x;
    const int f = threadIdx.x;
    float acc = __bfloat162float(in[c * HID + f]);
#pragma unroll
    for (int t = 0; t < TAPS; ++t) acc += Kw[f * TAPS + t] * __bfloat162float(in[nbr(c, nx, ny, t) * HID + f]);
    out[c * HID + f] = __float2bfloat16(acc);
}

// Backward of h_c = h + dwconv(h) followed by h = relu(z):
//   dh = dhc + conv^T(dhc), dz = dh * (h > 0)  (BF16, feeds the GEMMs)
// per block of RED_CHUNK columns: partial sums of dz (bias gradient) and of
// dhc[c] * h[nbr(c, t)] (kernel gradient), reduced later in block order.
__global__ void k_dwconv_bwd(const float *__restrict__ dhc, const bf16 *__restrict__ h, const float *__restrict__ Kw,
                             long long C, int nx, int ny, bf16 *__restrict__ dz, float *__restrict__ part_db,
                             float *__restrict__ part_dk) {
    const int f = threadIdx.x;
    const long long c0 = (long long)blockIdx.x * RED_CHUNK;
    float db = 0.f, dk[TAPS];
#pragma unroll
    for (int t = 0; t < TAPS; ++t) dk[t] = 0.f;
    for (long long c = c0; c < c0 + RED_CHUNK && c < C; ++c) {
        float dh = dhc[c * HID + f];
#pragma unroll
        for (int t = 0; t < TAPS; ++t) {
            // conv^T: the tap t of column nbr(c, 8 - t) reaches c
            dh += Kw[f * TAPS + (TAPS - 1 - t)] * dhc[nbr(c, nx, ny, t) * HID + f];
            dk[t] += dhc[c * HID + f] * __bfloat162float(h[nbr(c, nx, ny, t) * HID + f]);
        }
        const float z = __bfloat162float(h[c * HID + f]) > 0.f ? dh : 0.f;
        dz[c * HID + f] = __float2bfloat16(z);
        db += z;
    }
    part_db[(long long)blockIdx.x * HID + f] = db;
#pragma unroll
    for (int t = 0; t < TAPS; ++t) part_dk[((long long)blockIdx.x * HID + f) * TAPS + t] = dk[t];
}

// sum over the first dimension: out[j] = sum_b in[b * n + j] (fixed order)
__global__ void k_sum_rows(const float *__restrict__ in, int rows, int n, float *__restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    float acc = 0.f;
    for (int b = 0; b < rows; ++b) acc += in[(long long)b * n + j];
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

__global__ void k_loss_final(const double *__restrict__ part, int nb, double *__restrict__ scal) {
    double a = 0, b = 0;
    for (int i = 0; i < nb; ++i) {
        a += part[2 * i];
        b += part[2 * i + 1];
    }
    scal[0] = a;
    scal[1] = b;
    scal[2] = b > 0 ? a / b : a;
}

// dL/dY = 2 (Y - T) / sum T^2 (FP32 and BF16), and its column sums for db3
__global__ void k_dy(const float *__restrict__ Y, const float *__restrict__ T, long long n,
                     const double *__restrict__ scal, float *__restrict__ dyf, bf16 *__restrict__ dyb) {
    const double w = scal[1] > 0 ? 2.0 / scal[1] : 2.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float g = (float)(w * ((double)Y[i] - (double)T[i]));
        dyf[i] = g;
        dyb[i] = __float2bfloat16(g);
    }
}

// column sums of a [C][L] FP32 array, per block of RED_CHUNK columns
__global__ void k_colsum_part(const float *__restrict__ a, long long C, int F, float *__restrict__ part) {
    const int f = threadIdx.x;
    const long long c0 = (long long)blockIdx.x * RED_CHUNK;
    float acc = 0.f;
    for (long long c = c0; c < c0 + RED_CHUNK && c < C; ++c) acc += a[c * F + f];
    part[(long long)blockIdx.x * F + f] = acc;
}

// Adam (FP32 master weights), then refresh the BF16 copies of W1, W2, W3
__device__ __forceinline__ bool is_bias(int i) {
    return (i >= OFF_B1 && i < OFF_B1 + HID) || (i >= OFF_B2 && i < OFF_B2 + HID) || (i >= OFF_B3 && i < OFF_B3 + L);
}

__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, int n, float lr, float b1, float b2, float eps, float c1, float c2,
                       bf16 *__restrict__ w1b, bf16 *__restrict__ w2b, bf16 *__restrict__ w3b, int no_bias) {
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
    if (i >= OFF_W1 && i < OFF_W1 + HID * L) w1b[i - OFF_W1] = __float2bfloat16(pi);
    if (i >= OFF_W2 && i < OFF_W2 + HID * HID) w2b[i - OFF_W2] = __float2bfloat16(pi);
    if (i >= OFF_W3 && i < OFF_W3 + L * HID) w3b[i - OFF_W3] = __float2bfloat16(pi);
}

__global__ void k_params_to_bf16(const float *__restrict__ p, bf16 *__restrict__ w1b, bf16 *__restrict__ w2b,
                                 bf16 *__restrict__ w3b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < HID * L) w1b[i] = __float2bfloat16(p[OFF_W1 + i]);
    if (i < HID * HID) w2b[i] = __float2bfloat16(p[OFF_W2 + i]);
    if (i < L * HID) w3b[i] = __float2bfloat16(p[OFF_W3 + i]);
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

// Forward on the columns already gathered into net->x0 (C columns).
static int forward(Net *n, long long C, int nx, int ny) {
    cudaStream_t st = n->stream;
    int rc;
    umma::GemmArgs g = gargs((int)C, HID, L, n->x0, L, 1, n->w1b, L, 1, n->err);
    g.bias = n->param + OFF_B1;
    g.relu = 1;
    g.outB = n->h1;
    if ((rc = gemm(g, 1, st))) return rc;
    k_dwconv<<<(unsigned)C, HID, 0, st>>>(n->h1, n->param + OFF_K1, nx, ny, n->h1c);
    g = gargs((int)C, HID, HID, n->h1c, HID, 1, n->w2b, HID, 1, n->err);
    g.bias = n->param + OFF_B2;
    g.relu = 1;
    g.outB = n->h2;
    if ((rc = gemm(g, 1, st))) return rc;
    k_dwconv<<<(unsigned)C, HID, 0, st>>>(n->h2, n->param + OFF_K2, nx, ny, n->h2c);
    g = gargs((int)C, L, HID, n->h2c, HID, 1, n->w3b, HID, 1, n->err);
    g.bias = n->param + OFF_B3;
    g.outF = n->y;
    if ((rc = gemm(g, 1, st))) return rc;
    PCF_CUDA_TRY(cudaGetLastError());
    return PCF_OK;
}

// Loss and gradients (into n->grad) for targets already gathered into n->t.
static int backward(Net *n, long long C, int nx, int ny) {
    cudaStream_t st = n->stream;
    int rc;
    const long long ny_ = C * L;
    const int nb = 256;
    k_loss_part<<<nb, 256, 0, st>>>(n->y, n->t, ny_, reinterpret_cast<double *>(n->red));
    k_loss_final<<<1, 1, 0, st>>>(reinterpret_cast<double *>(n->red), nb, n->scal);
    k_dy<<<1024, 256, 0, st>>>(n->y, n->t, ny_, n->scal, n->dyf, n->dyb);
    const unsigned nchunk = (unsigned)((C + RED_CHUNK - 1) / RED_CHUNK);
    float *part_db = n->part, *part_dk = n->part + (long long)nchunk * HID;
    // b3
    k_colsum_part<<<nchunk, L, 0, st>>>(n->dyf, C, L, part_db);
    k_sum_rows<<<1, L, 0, st>>>(part_db, (int)nchunk, L, n->grad + OFF_B3);
    // W3 = dY^T h2c : [L][HID], K = C
    umma::GemmArgs g = gargs(L, HID, (int)C, n->dyb, 1, L, n->h2c, 1, HID, n->err);
    g.outF = n->part;
    if ((rc = gemm(g, KSPLIT, st))) return rc;
    k_sum_rows<<<(L * HID + 255) / 256, 256, 0, st>>>(n->part, std::min<int>(KSPLIT, (int)((C + 63) / 64)),
                                                       L * HID, n->grad + OFF_W3);
    // dh2c = dY W3 : [C][HID]
    g = gargs((int)C, HID, L, n->dyb, L, 1, n->w3b, 1, HID, n->err);
    g.outF = n->dh2c;
    if ((rc = gemm(g, 1, st))) return rc;
    // conv2 / relu2 backward -> dz2, b2, K2
    k_dwconv_bwd<<<nchunk, HID, 0, st>>>(n->dh2c, n->h2, n->param + OFF_K2, C, nx, ny, n->dz2, part_db, part_dk);
    k_sum_rows<<<1, HID, 0, st>>>(part_db, (int)nchunk, HID, n->grad + OFF_B2);
    k_sum_rows<<<(HID * TAPS + 255) / 256, 256, 0, st>>>(part_dk, (int)nchunk, HID * TAPS, n->grad + OFF_K2);
    // W2 = dz2^T h1c : [HID][HID]
    g = gargs(HID, HID, (int)C, n->dz2, 1, HID, n->h1c, 1, HID, n->err);
    g.outF = n->part;
    if ((rc = gemm(g, KSPLIT, st))) return rc;
    k_sum_rows<<<(HID * HID + 255) / 256, 256, 0, st>>>(n->part, std::min<int>(KSPLIT, (int)((C + 63) / 64)),
                                                         HID * HID, n->grad + OFF_W2);
    // dh1c = dz2 W2
    g = gargs((int)C, HID, HID, n->dz2, HID, 1, n->w2b, 1, HID, n->err);
    g.outF = n->dh1c;
    if ((rc = gemm(g, 1, st))) return rc;
    // conv1 / relu1 backward -> dz1, b1, K1
    k_dwconv_bwd<<<nchunk, HID, 0, st>>>(n->dh1c, n->h1, n->param + OFF_K1, C, nx, ny, n->dz1, part_db, part_dk);
    k_sum_rows<<<1, HID, 0, st>>>(part_db, (int)nchunk, HID, n->grad + OFF_B1);
    k_sum_rows<<<(HID * TAPS + 255) / 256, 256, 0, st>>>(part_dk, (int)nchunk, HID * TAPS, n->grad + OFF_K1);
    // W1 = dz1^T x0 : [HID][L]
    g = gargs(HID, L, (int)C, n->dz1, 1, HID, n->x0, 1, L, n->err);
    g.outF = n->part;
    if ((rc = gemm(g, KSPLIT, st))) return rc;
    k_sum_rows<<<(HID * L + 255) / 256, 256, 0, st>>>(n->part, std::min<int>(KSPLIT, (int)((C + 63) / 64)), HID * L,
                                                       n->grad + OFF_W1);
    PCF_CUDA_TRY(cudaGetLastError());
    return PCF_OK;
}

static int check_err(Net *n) {
    int e = 0;
    PCF_CUDA_TRY(cudaMemcpyAsync(&e, n->err, sizeof(int), cudaMemcpyDeviceToHost, n->stream));
    PCF_CUDA_TRY(cudaStreamSynchronize(n->stream));
    return e ? PCF_ECUDA : PCF_OK;
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

// deterministic parameter initialisation: He-uniform weights, zero biases,
// zero convolution kernels (so the network starts as a plain MLP)
void init_params(std::vector<float> &p, unsigned seed) {
    using namespace pcf::net;
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
    fill(OFF_W1, HID * L, L);
    fill(OFF_W2, HID * HID, HID);
    fill(OFF_W3, L * HID, HID);
    for (int i = 0; i < L * HID; ++i) p[OFF_W3 + i] *= 0.1f;  // small initial output
}

int net_alloc(pcf::net::Net &n, long long cap) {
    using namespace pcf::net;
    auto A = [&](void **q, size_t b) -> int {
        const cudaError_t e = cudaMalloc(q, b);
        return e == cudaSuccess ? PCF_OK : pcf_set_cuda_error(e);
    };
    const size_t f4 = sizeof(float), b2 = sizeof(bf16);
    const long long nchunk = (cap + RED_CHUNK - 1) / RED_CHUNK;
    const size_t part = std::max<size_t>((size_t)KSPLIT * HID * HID, (size_t)nchunk * HID * (TAPS + 1));
    int rc;
    if ((rc = A((void **)&n.param, NPARAM * f4)) || (rc = A((void **)&n.grad, NPARAM * f4)) ||
        (rc = A((void **)&n.m, NPARAM * f4)) || (rc = A((void **)&n.v, NPARAM * f4)) ||
        (rc = A((void **)&n.w1b, HID * L * b2)) || (rc = A((void **)&n.w2b, HID * HID * b2)) ||
        (rc = A((void **)&n.w3b, L * HID * b2)) || (rc = A((void **)&n.x0, cap * L * b2)) ||
        (rc = A((void **)&n.h1, cap * HID * b2)) || (rc = A((void **)&n.h1c, cap * HID * b2)) ||
        (rc = A((void **)&n.h2, cap * HID * b2)) || (rc = A((void **)&n.h2c, cap * HID * b2)) ||
        (rc = A((void **)&n.dyb, cap * L * b2)) || (rc = A((void **)&n.dz2, cap * HID * b2)) ||
        (rc = A((void **)&n.dz1, cap * HID * b2)) || (rc = A((void **)&n.y, cap * L * f4)) ||
        (rc = A((void **)&n.t, cap * L * f4)) || (rc = A((void **)&n.dyf, cap * L * f4)) ||
        (rc = A((void **)&n.dh2c, cap * HID * f4)) || (rc = A((void **)&n.dh1c, cap * HID * f4)) ||
        (rc = A((void **)&n.part, part * f4)) || (rc = A((void **)&n.red, 1024 * sizeof(double))) ||
        (rc = A((void **)&n.scal, 4 * sizeof(double))) || (rc = A((void **)&n.err, sizeof(int))))
        return rc;
    return PCF_OK;
}

int net_upload_params(pcf::net::Net &n, const float *host) {
    using namespace pcf::net;
    PCF_CUDA_TRY(cudaMemcpyAsync(n.param, host, NPARAM * sizeof(float), cudaMemcpyHostToDevice, n.stream));
    k_params_to_bf16<<<(HID * HID + 255) / 256, 256, 0, n.stream>>>(n.param, n.w1b, n.w2b, n.w3b);
    PCF_CUDA_TRY(cudaGetLastError());
    PCF_CUDA_TRY(cudaStreamSynchronize(n.stream));
    return PCF_OK;
}

template <typename T>
int net_gather(pcf::net::Net &n, const T *field, long long plane, int nz, float scale, float *dstF, bf16 *dstB) {
    using namespace pcf::net;
    const long long total = plane * L;
    const unsigned grid = (unsigned)((total + 255) / 256);
    if (dstB) k_gather<T, bf16><<<grid, 256, 0, n.stream>>>(field, plane, nz, scale, dstB);
    if (dstF) k_gather<T, float><<<grid, 256, 0, n.stream>>>(field, plane, nz, scale, dstF);
    PCF_CUDA_TRY(cudaGetLastError());
    return PCF_OK;
}

}  // namespace

extern "C" {

int pcf_net_num_params(void) { return pcf::net::NPARAM; }

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
        cudaMemsetAsync(w->n.m, 0, pcf::net::NPARAM * sizeof(float), w->n.stream);
        cudaMemsetAsync(w->n.v, 0, pcf::net::NPARAM * sizeof(float), w->n.stream);
        cudaMemsetAsync(w->n.grad, 0, pcf::net::NPARAM * sizeof(float), w->n.stream);
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
    pcf::net::Net &n = w->n;
    cudaSetDevice(n.device);
    void *ptrs[] = {n.param, n.grad, n.m, n.v, n.w1b, n.w2b, n.w3b, n.x0, n.h1, n.h1c, n.h2, n.h2c,
                    n.dyb, n.dz2, n.dz1, n.y, n.t, n.dyf, n.dh2c, n.dh1c, n.part, n.red, n.scal, n.err};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    if (n.stream) cudaStreamDestroy(n.stream);
    delete w;
    return PCF_OK;
}

int pcf_net_get_params(pcf_net *w, float *host) {
    if (!w || !host) return PCF_EINVAL;
    PCF_CUDA_TRY(cudaSetDevice(w->n.device));
    PCF_CUDA_TRY(cudaMemcpy(host, w->n.param, pcf::net::NPARAM * sizeof(float), cudaMemcpyDeviceToHost));
    return PCF_OK;
}

int pcf_net_set_params(pcf_net *w, const float *host) {
    if (!w || !host) return PCF_EINVAL;
    PCF_CUDA_TRY(cudaSetDevice(w->n.device));
    w->n.step = 0;
    cudaMemsetAsync(w->n.m, 0, pcf::net::NPARAM * sizeof(float), w->n.stream);
    cudaMemsetAsync(w->n.v, 0, pcf::net::NPARAM * sizeof(float), w->n.stream);
    return net_upload_params(w->n, host);
}

// Network output for a device field: out = beta * out + scale_out * N(scale_in * in).
// in / out: nz x ny x nx (x fastest), device memory; double or float by `fp64`.
int pcf_net_apply_device(pcf_net *w, const void *in, int nx, int ny, int nz, double scale_in, double scale_out,
                         double beta, void *out, int fp64, void *stream) {
    if (!w || !in || !out || nx < 1 || ny < 1 || nz < 1) return PCF_EINVAL;
    pcf::net::Net &n = w->n;
    const long long plane = (long long)nx * ny;
    if (plane > n.cap) return PCF_ERANGE;
    cudaStream_t caller = static_cast<cudaStream_t>(stream);
    cudaStream_t keep = n.stream;
    if (caller) n.stream = caller;  // run on the caller's stream
    int rc = fp64 ? net_gather<double>(n, (const double *)in, plane, nz, (float)scale_in, nullptr, n.x0)
                  : net_gather<float>(n, (const float *)in, plane, nz, (float)scale_in, nullptr, n.x0);
    if (!rc) rc = pcf::net::forward(&n, plane, nx, ny);
    if (!rc) {
        const unsigned grid = (unsigned)((plane * nz + 255) / 256);
        if (fp64)
            pcf::net::k_scatter<double><<<grid, 256, 0, n.stream>>>(n.y, plane, nz, (float)scale_out, (float)beta,
                                                                   (double *)out);
        else
            pcf::net::k_scatter<float><<<grid, 256, 0, n.stream>>>(n.y, plane, nz, (float)scale_out, (float)beta,
                                                                  (float *)out);
        if (cudaGetLastError() != cudaSuccess) rc = PCF_ECUDA;
    }
    n.stream = keep;
    return rc;
}

int pcf_net_set_bias_free(pcf_net *w, int on) {
    if (!w) return PCF_EINVAL;
    using namespace pcf::net;
    Net &n = w->n;
    PCF_CUDA_TRY(cudaSetDevice(n.device));
    n.no_bias = on ? 1 : 0;
    if (on) {
        const int offs[3] = {OFF_B1, OFF_B2, OFF_B3}, lens[3] = {HID, HID, L};
        for (int q = 0; q < 3; ++q)
            for (float *a : {n.param, n.m, n.v})
                PCF_CUDA_TRY(cudaMemsetAsync(a + offs[q], 0, sizeof(float) * lens[q], n.stream));
        PCF_CUDA_TRY(cudaStreamSynchronize(n.stream));
    }
    return PCF_OK;
}

// Host-array forward (tests): out = N(in), both nz x ny x nx doubles.
int pcf_net_forward(pcf_net *w, const double *in, int nx, int ny, int nz, double *out) {
    if (!w || !in || !out) return PCF_EINVAL;
    PCF_CUDA_TRY(cudaSetDevice(w->n.device));
    const size_t bytes = sizeof(double) * (size_t)nx * ny * nz;
    double *d = nullptr;
    PCF_CUDA_TRY(cudaMalloc(&d, 2 * bytes));
    int rc = PCF_OK;
    if (cudaMemcpy(d, in, bytes, cudaMemcpyHostToDevice) != cudaSuccess) rc = PCF_ECUDA;
    if (!rc) rc = pcf_net_apply_device(w, d, nx, ny, nz, 1.0, 1.0, 0.0, d + (size_t)nx * ny * nz, 1, nullptr);
    if (!rc && cudaStreamSynchronize(w->n.stream) != cudaSuccess) rc = PCF_ECUDA;
    if (!rc) rc = pcf::net::check_err(&w->n);
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
    using namespace pcf::net;
    if (!w || !b || !x || nx < 1 || ny < 1 || nz < 1) return PCF_EINVAL;
    Net &n = w->n;
    const long long plane = (long long)nx * ny;
    if (plane > n.cap) return PCF_ERANGE;
    PCF_CUDA_TRY(cudaSetDevice(n.device));
    int rc = net_gather<float>(n, b, plane, nz, 1.0f, nullptr, n.x0);
    if (!rc) rc = net_gather<float>(n, x, plane, nz, 1.0f, n.t, nullptr);
    if (!rc) rc = forward(&n, plane, nx, ny);
    if (!rc) rc = backward(&n, plane, nx, ny);
    if (rc) return rc;
    if (lr > 0) {
        n.step += 1;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - std::pow(b1, (float)n.step), c2 = 1.f - std::pow(b2, (float)n.step);
        k_adam<<<(NPARAM + 255) / 256, 256, 0, n.stream>>>(n.param, n.grad, n.m, n.v, NPARAM, (float)lr, b1, b2,
                                                           1e-8f, c1, c2, n.w1b, n.w2b, n.w3b, n.no_bias);
        PCF_CUDA_TRY(cudaGetLastError());
    }
    double s[3];
    PCF_CUDA_TRY(cudaMemcpyAsync(s, n.scal, sizeof(s), cudaMemcpyDeviceToHost, n.stream));
    if (grad) PCF_CUDA_TRY(cudaMemcpyAsync(grad, n.grad, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, n.stream));
    PCF_CUDA_TRY(cudaStreamSynchronize(n.stream));
    if ((rc = check_err(&n))) return rc;
    if (loss) *loss = s[2];
    return PCF_OK;
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

// Weights file: "PCFNET01", int32 NPARAM, int32 Adam step, then NPARAM FP32 values.
int pcf_net_save(pcf_net *w, const char *path) {
    if (!w || !path) return PCF_EINVAL;
    std::vector<float> p(pcf::net::NPARAM);
    int rc = pcf_net_get_params(w, p.data());
    if (rc) return rc;
    FILE *f = std::fopen(path, "wb");
    if (!f) return PCF_EINVAL;
    const int hdr[2] = {pcf::net::NPARAM, w->n.step};
    const bool ok = std::fwrite("PCFNET01", 1, 8, f) == 8 && std::fwrite(hdr, sizeof(int), 2, f) == 2 &&
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
    std::vector<float> p(pcf::net::NPARAM);
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "PCFNET01", 8) == 0 &&
              std::fread(hdr, sizeof(int), 2, f) == 2 && hdr[0] == pcf::net::NPARAM &&
              std::fread(p.data(), sizeof(float), p.size(), f) == p.size();
    std::fclose(f);
    if (!ok) return PCF_EINVAL;
    return pcf_net_set_params(w, p.data());
}

}  // extern "C"
