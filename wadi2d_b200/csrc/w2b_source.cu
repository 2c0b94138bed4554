// Sources and books on the device: the rain excess of a source window per cell (FP64, written to src as float32),
// and the FP64 storage of a set of cells. Both reductions run in a fixed order (per-block tree, then one block over
// the partials), so a result does not depend on scheduling.
//
// The rate restates wadi2d/forcing.py:667-683 per cell: excess = (E(P1) - E(P0)) / (1000 dt), with the SCS loss of
// wadi2d/hydrology/losses.py:69-72 or the initial-and-constant loss of wadi2d_b200/forcing.py; the window's rain
// volume is the sum of the float32 rates times the cell area in FP64, times dt. The lumped inflows restate the inflow
// part of wadi2d/forcing.py:684-694 with the depths read in place. Storage restates
// wadi2d/engine/monitor.py:214-218 (h + res over the interior cells, FP64). Each cell is weighed by the area of its
// run's cells and its mean depth read from its run's current half, so one call serves a batch of runs as well.
#include <cstdio>
#include <cstring>

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

// numpy's pairwise summation of n doubles (np.add.reduce on a contiguous float64 array, numpy's pairwise_sum): fewer
// than 8 terms added in order from 0; up to 128 in eight interleaved partial sums combined as ((r0 + r1) + (r2 + r3)) +
// ((r4 + r5) + (r6 + r7)), then the tail in order; beyond 128 the two halves (the first a multiple of 8 long) summed
// so and added. Restated so that a device sum rounds as the host's np.sum does. Recursion unrolled with a stack.
__device__ double pairwise_sum(const double* a, int n) {
    struct Span {
        int at, n, state;
        double left;
    };
    Span stack[32];
    int top = 0;
    stack[0] = {0, n, 0, 0.0};
    double ret = 0.0;
    while (top >= 0) {
        Span& sp = stack[top];
        if (sp.n <= 128) {
            double res;
            const double* x = a + sp.at;
            if (sp.n < 8) {
                res = 0.0;
                for (int i = 0; i < sp.n; ++i) res += x[i];
            } else {
                double r[8];
                for (int j = 0; j < 8; ++j) r[j] = x[j];
                int i = 8;
                for (; i < sp.n - (sp.n % 8); i += 8)
                    for (int j = 0; j < 8; ++j) r[j] += x[i + j];
                res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
                for (; i < sp.n; ++i) res += x[i];
            }
            ret = res;
            --top;
            continue;
        }
        int n2 = sp.n / 2;
        n2 -= n2 % 8;
        if (sp.state == 0) {  // the first half
            sp.state = 1;
            stack[top + 1] = {sp.at, n2, 0, 0.0};
            ++top;
        } else if (sp.state == 1) {  // the first half's sum came back: now the second
            sp.left = ret;
            sp.state = 2;
            stack[top + 1] = {sp.at + n2, sp.n - n2, 0, 0.0};
            ++top;
        } else {
            ret = sp.left + ret;
            --top;
        }
    }
    return ret;
}

// The lumped inflows of a source window (wadi2d/forcing.py:684-694), in the host's order, one CTA: first every
// injection cell's source is reset to the window's rain rate where the rain pass wrote one (else 0); then injection
// by injection, those with a positive mean flow q share it over their cells (Injection.share,
// wadi2d/forcing.py:468-476): by the level d read in place where d >= the injection's minimum depth, all to its
// lowest cell while none is, the weights summed as np.sum sums them; each cell's float32 rate (q share / area) is
// added to src as the host adds it; the injection's window volume is the float32 rates summed in FP64 (np.sum's
// order) times the area and the window, and the window's total is added to volume[n].
// The per-injection numbers of a window, by value: the mean flows, the cell ranges, the lowest cells and the depth
// floors (all checked on the host).
struct InflowArgs {
    int32_t n, start[W2B_INFLOWS_MAX + 1], lowest[W2B_INFLOWS_MAX];
    double q[W2B_INFLOWS_MAX], min_depth[W2B_INFLOWS_MAX];
    double area;
    const int32_t* cells;
    const uint8_t* rained;
    double* volume;
};

__global__ void __launch_bounds__(256) inflow_kernel(StepArgs A, InflowArgs F, double step) {
    __shared__ double w[W2B_INFLOW_CELLS_MAX];
    float* src = const_cast<float*>(A.src);
    const int tid = threadIdx.x;
    const int all = F.start[F.n];
    for (int j = tid; j < all; j += blockDim.x) {
        const int k = F.cells[j];
        if (!F.rained[j]) src[k] = 0.0f;
    }
    __syncthreads();
    double total = 0.0;
    for (int i = 0; i < F.n; ++i) {
        const double q = F.q[i];
        const int s = F.start[i], m = F.start[i + 1] - s;
        if (!(q > 0.0)) {
            if (tid == 0) F.volume[i] = 0.0;
            continue;
        }
        const double floor_depth = F.min_depth[i];
        int wet = 0;
        for (int j = tid; j < m; j += blockDim.x) {
            const double dj = (double)A.d[F.cells[s + j]];
            const bool on = dj >= floor_depth;
            w[j] = on ? dj : 0.0;
            wet |= on;
        }
        wet = __syncthreads_or(wet);
        if (tid == 0) {
            const double sum = wet ? pairwise_sum(w, m) : 0.0;
            for (int j = 0; j < m; ++j) {
                const double share = wet ? w[j] / sum : (j == F.lowest[i] ? 1.0 : 0.0);
                const float rate = (float)(q * share / F.area);
                const int k = F.cells[s + j];
                src[k] = src[k] + rate;
                w[j] = (double)rate;
            }
            const double vol = pairwise_sum(w, m) * F.area * step;
            F.volume[i] = vol;
            total += vol;
        }
        __syncthreads();
    }
    if (tid == 0) F.volume[F.n] += total;
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

int32_t w2b_inflow_window(void* handle, const W2BInflow* inflow, const double* q, double t0, double t1,
                          void* stream) {
    if (!handle || !inflow || !(t1 > t0) || inflow->n < 0 || inflow->n > W2B_INFLOWS_MAX || (inflow->n && !q) ||
        !inflow->volume || !(inflow->area > 0.0) ||
        (inflow->n && (!inflow->start || !inflow->cells || !inflow->lowest || !inflow->min_depth || !inflow->rained)))
        return W2B_EINVAL;
    InflowArgs F;
    memset(&F, 0, sizeof(F));
    F.n = inflow->n;
    F.area = inflow->area;
    F.cells = inflow->cells;
    F.rained = inflow->rained;
    F.volume = inflow->volume;
    if (F.n && inflow->start[0] != 0) return W2B_EINVAL;
    for (int i = 0; i < F.n; ++i) {
        const int m = inflow->start[i + 1] - inflow->start[i];
        if (m < 1 || m > W2B_INFLOW_CELLS_MAX || inflow->lowest[i] < 0 || inflow->lowest[i] >= m) return W2B_EINVAL;
        F.start[i] = inflow->start[i];
        F.lowest[i] = inflow->lowest[i];
        F.q[i] = q[i];
        F.min_depth[i] = inflow->min_depth[i];
    }
    F.start[F.n] = F.n ? inflow->start[F.n] : 0;
    StepArgs A;
    if (!handle_args(handle, &A)) return W2B_EINVAL;
    inflow_kernel<<<1, 256, 0, (cudaStream_t)stream>>>(A, F, t1 - t0);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "libwadi_b200: w2b_inflow_window: %s\n", cudaGetErrorString(e));
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
