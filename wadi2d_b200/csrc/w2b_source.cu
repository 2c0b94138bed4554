// Sources and books on the device: the rain excess of a source window per cell (FP64, written to src as float32),
// and the FP64 storage of a set of cells. Both reductions run in a fixed order (per-block tree, then one block over
// the partials), so a result does not depend on scheduling.
//
// The rate restates wadi2d/forcing.py:667-683 per cell: excess = (E(P1) - E(P0)) / (1000 dt), with the SCS loss of
// wadi2d/hydrology/losses.py:69-72 or the initial-and-constant loss of wadi2d_b200/forcing.py; the window's rain
// volume is the sum of the float32 rates times the cell area in FP64, times dt. Storage restates
// wadi2d/engine/monitor.py:214-218 (h + res over the interior cells, FP64). Each cell is weighed by the area of its
// run's cells and its mean depth read from its run's current half, so one call serves a batch of runs as well.
#include <cstdio>

#include "w2b_common.cuh"

namespace w2b {

constexpr int SRC_BLOCKS = 296;
constexpr int SRC_THREADS = 256;

__device__ __forceinline__ double block_sum(double v, double* red) {
    red[threadIdx.x] = v;
    __syncthreads();
    for (int s = SRC_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    return red[0];
}

// The cell area of NATIVE index k's run.
__device__ __forceinline__ double cell_area(const StepArgs& A, int k) {
    const double dx = (double)A.R.dx[A.tile_run[tile_of_native(A, k)]];
    return dx * dx;
}

__global__ void __launch_bounds__(SRC_THREADS) rain_kernel(StepArgs A, W2BRain R, double f0, double f1, double dt) {
    float* src = const_cast<float*>(A.src);
    __shared__ double red[SRC_THREADS];
    double acc = 0.0;
    for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < R.n; m += (int64_t)gridDim.x * blockDim.x) {
        const double D = R.depth[m];
        const double p0 = D * f0, p1 = D * f1;
        double mm;
        if (R.loss == 1) {
            // SCS: Pe(P) = (P - Ia)^2 / (P - Ia + S), zero up to Ia
            const double ia = R.ia_mm[m], s = R.s_mm[m];
            const double e0 = p0 - ia > 0.0 ? p0 - ia : 0.0;
            const double e1 = p1 - ia > 0.0 ? p1 - ia : 0.0;
            double x0 = e0 * e0 / (e0 + s), x1 = e1 * e1 / (e1 + s);
            x0 = isfinite(x0) ? x0 : 0.0;
            x1 = isfinite(x1) ? x1 : 0.0;
            mm = x1 - x0;
        } else if (R.loss == 2) {
            // initial loss first, then the constant rate over the rest of the window
            const double p = p1 - p0;
            const double left = R.ia_mm[m] - p0 > 0.0 ? R.ia_mm[m] - p0 : 0.0;
            const double after = p - left > 0.0 ? p - left : 0.0;
            const double share = p > 0.0 ? after / p : 0.0;
            const double x = after - R.fc_mm_h * share * dt / 3600.0;
            mm = x > 0.0 ? x : 0.0;
        } else {
            mm = p1 - p0;
        }
        const float rate = (float)(mm / (1000.0 * dt));
        const int k = R.cells[m];
        src[k] = rate;
        acc += (double)rate * cell_area(A, k);
    }
    const double b = block_sum(acc, red);
    if (threadIdx.x == 0) R.partial[blockIdx.x] = b;
}

__global__ void __launch_bounds__(SRC_THREADS) storage_kernel(StepArgs A, int64_t n, const int32_t* __restrict__ cells,
                                                              double* __restrict__ partial) {
    __shared__ double red[SRC_THREADS];
    double acc = 0.0;
    for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < n; m += (int64_t)gridDim.x * blockDim.x) {
        const int k = cells[m];
        const float* h = A.hh[A.R.parity[A.tile_run[tile_of_native(A, k)]]];
        acc += ((double)h[k] + (double)A.res[k]) * cell_area(A, k);
    }
    const double b = block_sum(acc, red);
    if (threadIdx.x == 0) partial[blockIdx.x] = b;
}

// src at each listed cell = its run's rate (a batch of runs under uniform rain of their own).
__global__ void __launch_bounds__(SRC_THREADS) source_runs_kernel(StepArgs A, int64_t n,
                                                                  const int32_t* __restrict__ cells,
                                                                  const float* __restrict__ rate) {
    float* src = const_cast<float*>(A.src);
    for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < n; m += (int64_t)gridDim.x * blockDim.x) {
        const int k = cells[m];
        src[k] = rate[A.tile_run[tile_of_native(A, k)]];
    }
}

// out[0] = scale * (sum of the partials, in order)
__global__ void __launch_bounds__(SRC_THREADS) finish_kernel(const double* __restrict__ partial, int n, double scale,
                                                             double* __restrict__ out) {
    __shared__ double red[SRC_THREADS];
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partial[i];
    const double b = block_sum(acc, red);
    if (threadIdx.x == 0) out[0] = b * scale;
}

}  // namespace w2b

using namespace w2b;

extern "C" {

int32_t w2b_rain_window(void* handle, const W2BRain* rain, double f0, double f1, double t0, double t1,
                        double* volume, void* stream) {
    if (!handle || !rain || !volume || !(t1 > t0) || rain->n < 0 || (rain->n && (!rain->cells || !rain->depth)) ||
        !rain->partial || (rain->loss == 1 && (!rain->s_mm || !rain->ia_mm)) || (rain->loss == 2 && !rain->ia_mm))
        return W2B_EINVAL;
    StepArgs A;
    if (!handle_args(handle, &A)) return W2B_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    const double dt = t1 - t0;
    rain_kernel<<<SRC_BLOCKS, SRC_THREADS, 0, s>>>(A, *rain, f0, f1, dt);
    finish_kernel<<<1, SRC_THREADS, 0, s>>>(rain->partial, SRC_BLOCKS, dt, volume);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "libwadi_b200: w2b_rain_window: %s\n", cudaGetErrorString(e));
        return W2B_ECUDA;
    }
    return W2B_OK;
}

int32_t w2b_source_runs(void* handle, int64_t n, const int32_t* cells, const float* rate, void* stream) {
    if (!handle || n < 0 || (n && (!cells || !rate))) return W2B_EINVAL;
    StepArgs A;
    if (!handle_args(handle, &A)) return W2B_EINVAL;
    if (n) source_runs_kernel<<<SRC_BLOCKS, SRC_THREADS, 0, (cudaStream_t)stream>>>(A, n, cells, rate);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "libwadi_b200: w2b_source_runs: %s\n", cudaGetErrorString(e));
        return W2B_ECUDA;
    }
    return W2B_OK;
}

int32_t w2b_storage(void* handle, int64_t n, const int32_t* cells, double* partial, double* out, void* stream) {
    if (!handle || n < 0 || (n && !cells) || !partial || !out) return W2B_EINVAL;
    StepArgs A;
    if (!handle_args(handle, &A)) return W2B_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    storage_kernel<<<SRC_BLOCKS, SRC_THREADS, 0, s>>>(A, n, cells, partial);
    finish_kernel<<<1, SRC_THREADS, 0, s>>>(partial, SRC_BLOCKS, 1.0, out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "libwadi_b200: w2b_storage: %s\n", cudaGetErrorString(e));
        return W2B_ECUDA;
    }
    return W2B_OK;
}

}  // extern "C"
