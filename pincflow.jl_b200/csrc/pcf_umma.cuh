// pcf_umma.cuh -- BF16 GEMM on the sm_100a tensor cores (tcgen05 / UMMA) for
// the dense layers of the learned preconditioner.
//
//   D[m, n] = sum_k A(m, k) B(n, k)      A(m,k) = A[m*a_rs + k*a_ks], B likewise
//
// One CTA of 128 threads computes a 128 x NT tile of D (NT = 64 or 256, the
// full N of the network's layers) over a range of K (split-K over gridDim.z).
// Per K step of 64 the CTA stages A (128 x 64) and B (NT x 64) in shared
// memory in the UMMA canonical K-major layout without swizzle (core matrices
// of 8 rows x 16 bytes stored contiguously; LBO = 128 B between core matrices
// adjacent in K, SBO = 1024 B between core matrices adjacent in M/N), one
// elected thread issues four tcgen05.mma (K = 16 each) into an FP32
// accumulator in tensor memory, and tcgen05.commit arrives on an mbarrier
// that all threads wait on (bounded).  The epilogue reads the accumulator
// with tcgen05.ld (warp w owns TMEM lanes 32w..32w+31 = rows) and applies
// bias / ReLU / split-K partial stores.  Descriptor bit layouts follow the
// sm100 UMMA SmemDescriptor and InstrDescriptor (kind::f16).
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

#include "pcf_internal.cuh"

namespace pcf {
namespace umma {

struct GemmArgs {
    int M, N, K;
    const __nv_bfloat16 *A;
    long long a_rs, a_ks;
    const __nv_bfloat16 *B;
    long long b_rs, b_ks;
    const float *bias;     // per column n (nullable; not with split-K)
    int relu;              // apply max(0, .) after the bias
    float *outF;           // row-major [M][ldo] FP32 (split-K: [gridDim.z][M][N] partials)
    __nv_bfloat16 *outB;   // row-major [M][ldo] BF16 (nullable)
    long long ldo;         // output row length (0: N); lets a launch write a column block of a wider matrix
    int *error;            // set to 1 if an mbarrier wait timed out
};

// Shared-memory matrix descriptor: K-major, SWIZZLE_NONE.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);        // start address, bits [0,14)
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;    // leading byte offset, bits [16,30)
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;    // stride byte offset, bits [32,46)
    d |= (uint64_t)1 << 46;                          // version = 1 (sm100), bits [46,48)
    return d;                                        // base offset 0, lbo mode 0, layout SWIZZLE_NONE (0)
}

// Instruction descriptor, kind::f16: BF16 x BF16 -> FP32, A and B K-major.
__host__ __device__ constexpr uint32_t instr_desc(int M, int N) {
    return (1u << 4)                                // D format F32, bits [4,6)
           | (1u << 7)                              // A format BF16, bits [7,10)
           | (1u << 10)                             // B format BF16, bits [10,13)
           | ((uint32_t)(N >> 3) << 17)             // N / 8, bits [17,23)
           | ((uint32_t)(M >> 4) << 24);            // M / 16, bits [24,29)
}

// byte offset of element (row, k) of a (rows x 64) K-major tile
__device__ __forceinline__ uint32_t tile_off(int row, int k) {
    return (uint32_t)((((row >> 3) << 3) + (k >> 3)) * 128 + ((row & 7) << 4) + ((k & 7) << 1));
}

template <int NT>
__global__ void __launch_bounds__(128) k_gemm_bf16(GemmArgs g) {
    static_assert(NT == 64 || NT == 128 || NT == 256, "NT");
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *sA = smem;                          // 128 x 64 bf16 = 16 KB
    uint8_t *sB = smem + 16384;                  // NT x 64 bf16
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + 16384 + NT * 128);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * 128;
    const int ksteps = (g.K + 63) / 64;
    const int per = (ksteps + gridDim.z - 1) / gridDim.z;
    const int s_lo = blockIdx.z * per;
    const int s_hi = min(ksteps, s_lo + per);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(NT));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tslot;
    constexpr uint32_t idesc = instr_desc(128, NT);
    const uint32_t a_base = smem_u32(sA), b_base = smem_u32(sB), mb = smem_u32(mbar);

    uint32_t phase = 0;
    bool ok = true;
    for (int s = s_lo; s < s_hi; ++s) {
        const int k0 = s * 64;
        // stage A and B; the loop order follows the unit-stride global index
        if (g.a_ks == 1) {
            for (int e = tid; e < 128 * 64; e += 128) {
                const int r = e >> 6, k = e & 63;
                const int gm = m0 + r, gk = k0 + k;
                const __nv_bfloat16 v = (gm < g.M && gk < g.K) ? g.A[gm * g.a_rs + gk] : __float2bfloat16(0.0f);
                *reinterpret_cast<__nv_bfloat16 *>(sA + tile_off(r, k)) = v;
            }
        } else {
            for (int e = tid; e < 128 * 64; e += 128) {
                const int k = e >> 7, r = e & 127;
                const int gm = m0 + r, gk = k0 + k;
                const __nv_bfloat16 v =
                    (gm < g.M && gk < g.K) ? g.A[gm * g.a_rs + (long long)gk * g.a_ks] : __float2bfloat16(0.0f);
                *reinterpret_cast<__nv_bfloat16 *>(sA + tile_off(r, k)) = v;
            }
        }
        if (g.b_ks == 1) {
            for (int e = tid; e < NT * 64; e += 128) {
                const int r = e >> 6, k = e & 63;
                const int gk = k0 + k;
                const __nv_bfloat16 v = (r < g.N && gk < g.K) ? g.B[r * g.b_rs + gk] : __float2bfloat16(0.0f);
                *reinterpret_cast<__nv_bfloat16 *>(sB + tile_off(r, k)) = v;
            }
        } else {
            for (int e = tid; e < NT * 64; e += 128) {
                const int k = e / NT, r = e % NT;
                const int gk = k0 + k;
                const __nv_bfloat16 v =
                    (r < g.N && gk < g.K) ? g.B[r * g.b_rs + (long long)gk * g.b_ks] : __float2bfloat16(0.0f);
                *reinterpret_cast<__nv_bfloat16 *>(sB + tile_off(r, k)) = v;
            }
        }
        // make the generic-proxy smem writes visible to the tensor core (async proxy)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
            for (int j = 0; j < 4; ++j) {  // K = 16 per instruction: advance two core matrices (256 B)
                const uint64_t da = smem_desc(a_base + j * 256, 128, 1024);
                const uint64_t db = smem_desc(b_base + j * 256, 128, 1024);
                const uint32_t acc = (s > s_lo || j > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mb)
                         : "memory");
        }
        if (!mbar_wait(mb, phase)) {
            ok = false;
            break;
        }
        phase ^= 1u;
        __syncthreads();  // all threads past the wait before the tiles are overwritten
    }
    if (!ok) {
        if (tid == 0 && g.error) atomicExch(g.error, 1);
        // give the in-flight MMAs one more bounded wait before releasing TMEM
        mbar_wait(mb, phase);
    }
    asm volatile("tcgen05.fence::after_thread_sync;");

    // epilogue: warp w reads TMEM lanes (rows) 32w .. 32w+31, 16 columns at a time
    const int row = m0 + warp * 32 + lane;
    const bool partial = gridDim.z > 1;
    const long long ldo = g.ldo > 0 ? g.ldo : g.N;
#pragma unroll 1
    for (int c0 = 0; c0 < NT; c0 += 16) {
        uint32_t v[16];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
            "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
              "=r"(v[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (ok && row < g.M && s_lo < s_hi) {
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int col = c0 + q;
                if (col >= g.N) continue;
                float d = __uint_as_float(v[q]);
                if (partial) {
                    g.outF[((long long)blockIdx.z * g.M + row) * g.N + col] = d;
                } else {
                    if (g.bias) d += g.bias[col];
                    if (g.relu) d = fmaxf(d, 0.0f);
                    if (g.outF) g.outF[(long long)row * ldo + col] = d;
                    if (g.outB) g.outB[(long long)row * ldo + col] = __float2bfloat16(d);
                }
            }
        } else if (ok && row < g.M && partial) {
            for (int q = 0; q < 16; ++q)
                if (c0 + q < g.N) g.outF[((long long)blockIdx.z * g.M + row) * g.N + c0 + q] = 0.0f;
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NT));
}

template <int NT>
constexpr int gemm_smem_bytes() {
    return 16384 + NT * 128 + 16;
}

}  // namespace umma
}  // namespace pcf
