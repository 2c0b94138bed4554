// The surrogate's network on the tensor cores: C = A B^T with BF16 operands and an FP32 accumulator in tensor memory
// (tcgen05.mma, kind::f16, one CTA a 128-row tile), and the element-wise kernels of training (activation, its
// gradient, transposes, the mean-square-error gradient, column sums, Adam).
//
// The GEMM: A is M x K and B is N x K, both row-major BF16 (K-major for the MMA); C is M x N row-major FP32, plus an
// optional bias per column. 16 <= N <= 256 with N % 16 == 0, K % 16 == 0. One CTA of 4 warps takes rows
// [128 b, 128 b + 128) (rows past M read as zero and are not written). K is staged in chunks of up to 128: the
// chunk's A and B rows are copied into shared memory in the canonical K-major layout without swizzle (8-row x 16-byte
// core matrices; a core matrix's next K chunk 128 B on, the next 8-row group (K chunk / 8) x 128 B on), thread 0
// issues one MMA per 16 of K against the accumulator in tensor memory and commits it to an mbarrier, and the CTA
// waits (bounded) before the next chunk overwrites the tiles. The epilogue reads the accumulator with
// tcgen05.ld.32x32b (warp w owns tensor-memory lanes 32 w .. 32 w + 31, one row each). Every wait is bounded; a wait
// that gives up sets the status word, waits once more for the MMAs in flight, frees the tensor memory and returns.
#include <cuda_bf16.h>

#include <cstdint>
#include <cstdio>

#include "w2b_common.cuh"
#include "w2b_tma.cuh"

namespace w2b {

constexpr int GEMM_M = 128;
constexpr int GEMM_KC = 128;  // K staged a chunk at a time
constexpr int GEMM_SMEM = (GEMM_M + 256) * GEMM_KC * 2 + 1024;

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    // shared-memory matrix descriptor: start address, leading and stride byte offsets (16-byte units), version 1 for
    // this architecture, no swizzle (cute/arch/mma_sm100_desc.hpp SmemDescriptor)
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__global__ void __launch_bounds__(128, 1) umma_gemm_kernel(const __nv_bfloat16* __restrict__ A,
                                                            const __nv_bfloat16* __restrict__ B,
                                                            const float* __restrict__ bias, float* __restrict__ C,
                                                            int M, int N, int K, int32_t* status) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * GEMM_M;
    uint8_t* sA = smem;
    uint8_t* sB = smem + GEMM_M * GEMM_KC * 2;
    uint32_t ncols = 32;
    while ((int)ncols < N) ncols <<= 1;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(ncols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;
    // instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, N / 8, M / 16
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(GEMM_M >> 4) << 24);
    uint32_t phase = 0;
    bool ok = true;
    for (int k0 = 0; k0 < K && ok; k0 += GEMM_KC) {
        const int kw = K - k0 < GEMM_KC ? K - k0 : GEMM_KC;  // this chunk's K, a multiple of 16
        const int kc = kw / 8;                              // 16-byte pieces of a row
        const uint32_t sbo = (uint32_t)kc * 128u;
        for (int idx = tid; idx < GEMM_M * kc; idx += blockDim.x) {
            const int r = idx / kc, c = idx - r * kc;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (m0 + r < M) v = *reinterpret_cast<const uint4*>(A + (size_t)(m0 + r) * K + k0 + c * 8);
            *reinterpret_cast<uint4*>(sA + (r >> 3) * sbo + c * 128 + (r & 7) * 16) = v;
        }
        for (int idx = tid; idx < N * kc; idx += blockDim.x) {
            const int r = idx / kc, c = idx - r * kc;
            const uint4 v = *reinterpret_cast<const uint4*>(B + (size_t)r * K + k0 + c * 8);
            *reinterpret_cast<uint4*>(sB + (r >> 3) * sbo + c * 128 + (r & 7) * 16) = v;
        }
        fence_proxy_async();  // these generic writes, before the tensor cores read the tiles
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
            for (int s = 0; s < kw / 16; ++s) {
                const uint64_t da = umma_desc(a0 + s * 256, 128, sbo);
                const uint64_t db = umma_desc(b0 + s * 256, 128, sbo);
                const uint32_t acc = (k0 > 0 || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(&bar))
                         : "memory");
        }
        ok = mbar_wait(&bar, phase);
        if (!ok) mbar_wait(&bar, phase);  // once more for the MMAs in flight before anything is freed
        phase ^= 1u;
        ok = !__syncthreads_or(!ok);
        tc_fence_after();
    }
    if (ok) {
        const int row = m0 + warp * 32 + lane;
        for (int c0 = 0; c0 < N; c0 += 8) {
            uint32_t v[8];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < M) {
                for (int j = 0; j < 8; ++j) {
                    const float x = __uint_as_float(v[j]) + (bias ? bias[c0 + j] : 0.0f);
                    C[(size_t)row * N + c0 + j] = x;
                }
            }
        }
    } else if (tid == 0) {
        atomicExch(status, W2B_ETIMEOUT);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
    }
}

// ------------------------------------------------------------------ element-wise kernels of training

// out = bf16(relu(z)) (relu = 1) or bf16(z) (relu = 0)
__global__ void bf16_act_kernel(const float* __restrict__ z, int64_t n, int relu, __nv_bfloat16* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float v = z[i];
        out[i] = __float2bfloat16_rn(relu && !(v > 0.0f) ? 0.0f : v);
    }
}

// dz = bf16(g * [z > 0])
__global__ void relu_back_kernel(const float* __restrict__ g, const float* __restrict__ z, int64_t n,
                                 __nv_bfloat16* __restrict__ dz) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        dz[i] = __float2bfloat16_rn(z[i] > 0.0f ? g[i] : 0.0f);
}

// xt (cols x rows) = x^T (x: rows x cols), BF16; zero-padded to rows_pad columns of xt
__global__ void transpose_bf16_kernel(const __nv_bfloat16* __restrict__ x, int rows, int cols, int rows_pad,
                                      __nv_bfloat16* __restrict__ xt) {
    __shared__ __nv_bfloat16 tile[32][33];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = r0 + j, c = c0 + threadIdx.x;
        tile[j][threadIdx.x] = (r < rows && c < cols) ? x[(size_t)r * cols + c] : __float2bfloat16_rn(0.0f);
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int c = c0 + j, r = r0 + threadIdx.x;
        if (c < cols && r < rows_pad) xt[(size_t)c * rows_pad + r] = tile[threadIdx.x][j];
    }
}

// dy = bf16(scale (y - t)) over the m valid rows (zero for padded rows), and the loss partials sum (y - t)^2 in FP64
__global__ void mse_grad_kernel(const float* __restrict__ y, const float* __restrict__ t, int m, int m_pad, int n,
                                float scale, __nv_bfloat16* __restrict__ dy, double* __restrict__ partial) {
    __shared__ double red[256];
    double acc = 0.0;
    const int64_t total = (int64_t)m_pad * n;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        float g = 0.0f;
        if (i / n < m) {
            const float d = y[i] - t[i];
            acc += (double)d * (double)d;
            g = scale * d;
        }
        dy[i] = __float2bfloat16_rn(g);
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// out[c] = sum over rows of bf16 x[r][c], FP32, rows in order
__global__ void colsum_kernel(const __nv_bfloat16* __restrict__ x, int rows, int cols, float* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float s = 0.0f;
    for (int r = 0; r < rows; ++r) s += __bfloat162float(x[(size_t)r * cols + c]);
    out[c] = s;
}

// Adam on FP32 weights (bias-corrected steps lr_t = lr sqrt(1 - b2^t) / (1 - b1^t)), and their BF16 copy. With
// lr_table, the step size is lr_table[*step], read on the device (a captured training step replays with each step's
// own size).
__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int64_t n, float lr_t, const float* __restrict__ lr_table,
                            const int64_t* __restrict__ step, float b1, float b2, float eps,
                            __nv_bfloat16* __restrict__ wb) {
    if (lr_table) lr_t = lr_table[*step];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr_t * mi / (sqrtf(vi) + eps);
        w[i] = wi;
        if (wb) wb[i] = __float2bfloat16_rn(wi);
    }
}

}  // namespace w2b

using namespace w2b;

extern "C" {

int32_t w2b_mma_gemm(const void* a, const void* b, int32_t m, int32_t n, int32_t k, const float* bias, float* c,
                     int32_t* status, void* stream) {
    if (!a || !b || !c || !status || m < 1 || n < 16 || n > 256 || n % 16 || k < 16 || k % 16) return W2B_EINVAL;
    if (((uintptr_t)a & 15) || ((uintptr_t)b & 15)) return W2B_EINVAL;
    if (cudaFuncSetAttribute(umma_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, GEMM_SMEM) != cudaSuccess)
        return W2B_ECUDA;
    const int grid = (m + GEMM_M - 1) / GEMM_M;
    umma_gemm_kernel<<<grid, 128, GEMM_SMEM, (cudaStream_t)stream>>>(
        static_cast<const __nv_bfloat16*>(a), static_cast<const __nv_bfloat16*>(b), bias, c, m, n, k, status);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "libwadi_b200: w2b_mma_gemm: %s\n", cudaGetErrorString(e));
        return W2B_ECUDA;
    }
    return W2B_OK;
}

int32_t w2b_bf16_act(const float* z, int64_t n, int32_t relu, void* out, void* stream) {
    if (!z || !out || n < 0) return W2B_EINVAL;
    bf16_act_kernel<<<296, 256, 0, (cudaStream_t)stream>>>(z, n, relu, static_cast<__nv_bfloat16*>(out));
    return cudaGetLastError() == cudaSuccess ? W2B_OK : W2B_ECUDA;
}

int32_t w2b_relu_back(const float* g, const float* z, int64_t n, void* dz, void* stream) {
    if (!g || !z || !dz || n < 0) return W2B_EINVAL;
    relu_back_kernel<<<296, 256, 0, (cudaStream_t)stream>>>(g, z, n, static_cast<__nv_bfloat16*>(dz));
    return cudaGetLastError() == cudaSuccess ? W2B_OK : W2B_ECUDA;
}

int32_t w2b_transpose_bf16(const void* x, int32_t rows, int32_t cols, int32_t rows_pad, void* xt, void* stream) {
    if (!x || !xt || rows < 1 || cols < 1 || rows_pad < rows) return W2B_EINVAL;
    const dim3 grid((cols + 31) / 32, (rows_pad + 31) / 32);
    transpose_bf16_kernel<<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>(
        static_cast<const __nv_bfloat16*>(x), rows, cols, rows_pad, static_cast<__nv_bfloat16*>(xt));
    return cudaGetLastError() == cudaSuccess ? W2B_OK : W2B_ECUDA;
}

int32_t w2b_mse_grad(const float* y, const float* t, int32_t m, int32_t m_pad, int32_t n, float scale, void* dy,
                     double* partial, void* stream) {
    if (!y || !t || !dy || !partial || m < 0 || m_pad < m || n < 1) return W2B_EINVAL;
    mse_grad_kernel<<<64, 256, 0, (cudaStream_t)stream>>>(y, t, m, m_pad, n, scale, static_cast<__nv_bfloat16*>(dy),
                                                          partial);
    return cudaGetLastError() == cudaSuccess ? W2B_OK : W2B_ECUDA;
}

int32_t w2b_colsum_bf16(const void* x, int32_t rows, int32_t cols, float* out, void* stream) {
    if (!x || !out || rows < 0 || cols < 1) return W2B_EINVAL;
    colsum_kernel<<<(cols + 127) / 128, 128, 0, (cudaStream_t)stream>>>(static_cast<const __nv_bfloat16*>(x), rows,
                                                                        cols, out);
    return cudaGetLastError() == cudaSuccess ? W2B_OK : W2B_ECUDA;
}

int32_t w2b_adam(float* w, const float* g, float* m, float* v, int64_t n, float lr_t, float b1, float b2, float eps,
                 void* wb, void* stream) {
    if (!w || !g || !m || !v || n < 0) return W2B_EINVAL;
    adam_kernel<<<296, 256, 0, (cudaStream_t)stream>>>(w, g, m, v, n, lr_t, nullptr, nullptr, b1, b2, eps,
                                                       static_cast<__nv_bfloat16*>(wb));
    return cudaGetLastError() == cudaSuccess ? W2B_OK : W2B_ECUDA;
}

int32_t w2b_adam_table(float* w, const float* g, float* m, float* v, int64_t n, const float* lr_table,
                       const int64_t* step, float b1, float b2, float eps, void* wb, void* stream) {
    if (!w || !g || !m || !v || !lr_table || !step || n < 0) return W2B_EINVAL;
    adam_kernel<<<296, 256, 0, (cudaStream_t)stream>>>(w, g, m, v, n, 0.0f, lr_table, step, b1, b2, eps,
                                                       static_cast<__nv_bfloat16*>(wb));
    return cudaGetLastError() == cudaSuccess ? W2B_OK : W2B_ECUDA;
}

}  // extern "C"
