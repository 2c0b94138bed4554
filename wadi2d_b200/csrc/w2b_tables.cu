// The sub-grid table builder on the GPU: every static array of the step from the bed's pixels.
//
// Restates wadi2d/tables/core.py (cell tables :16-41, face tables :44-79, local hydraulic radius :82-179 and
// :324-371, centre beds :267-279) and wadi2d/tables/builder.py (the per-tile windows :199-238, inverts, closed faces
// and natural crests :290-308) in FP64 with the reference's summation order: every running sum is taken by one
// thread in the reference's sequence, so the only difference from the CPU build is the last-ulp rounding of CUDA's
// double cbrt and pow against glibc's, which the float32 tables almost never see.
//
// Pixels are read from the whole bed with clipped indices, which is what the reference's per-tile windows of an
// ArrayBed hold (wadi2d/tables/builder.py:47-50): a window that reaches past the bed repeats its edge pixel.
#include <cmath>
#include <cstdio>
#include <mutex>

#include "w2b_common.cuh"

namespace w2b {

struct TableArgs {
    const double* z;
    int64_t zh, zw;
    int32_t roff, coff;
    const double* npix;  // per-pixel Manning n aligned with z (NaN: the cell's own), or null
    const double* nman;  // (ny, nx)
    const double *xcrest, *xlen, *xc, *ycrest, *ylen, *yc;  // (ny, nx)
    const uint8_t *xwall, *ywall, *mask;                    // (ny, nx); walls may be null
    const int32_t* tiles;
    int32_t ntiles, ny, nx, k, rows, local, margin, nmax;
    double pixel, e_lo, e_hi, beta, tol;
    // outputs, tile layout (ntiles, 32, 32[, rows[, 2]]) float32
    float *hc, *dtab, *efx, *efy, *ftabx, *ftaby, *zcx, *zcy;
    float *flx, *frx, *glx, *grx, *cwx, *fly, *fry, *gly, *gry, *cwy;
    // outputs, dense (ny, nx) float64
    double *zmin, *rel, *zfx, *zfy;
    // workspace of the local radius: 9 * (nmax + 1) doubles per thread of the face kernel
    double* ws;
    int64_t ws_threads;
};

__device__ __forceinline__ double zpix(const TableArgs& A, int64_t r, int64_t c) {
    r += A.roff;
    c += A.coff;
    r = r < 0 ? 0 : (r >= A.zh ? A.zh - 1 : r);
    c = c < 0 ? 0 : (c >= A.zw ? A.zw - 1 : c);
    return A.z[r * A.zw + c];
}

__device__ __forceinline__ double npix_at(const TableArgs& A, int64_t r, int64_t c) {
    r += A.roff;
    c += A.coff;
    r = r < 0 ? 0 : (r >= A.zh ? A.zh - 1 : r);
    c = c < 0 ? 0 : (c >= A.zw ? A.zw - 1 : c);
    return A.npix[r * A.zw + c];
}

__device__ __forceinline__ double lined(double pixel_n, double cell_n) {
    return isnan(pixel_n) ? 1.0 : cell_n / pixel_n;
}

// ------------------------------------------------------------------ cell tables (one thread per cell)

template <int K2MAX>
__global__ void __launch_bounds__(128) cell_tables_kernel(TableArgs A) {
    const int64_t ncell = (int64_t)(A.ntiles - 1) * TILE2;
    const int k = A.k, n = k * k, rows = A.rows, last = rows - 1;
    double p[K2MAX];
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += (int64_t)gridDim.x * blockDim.x) {
        const int t = (int)(c / TILE2) + 1;
        const int local = (int)(c % TILE2);
        const int64_t j = (int64_t)A.tiles[2 * t] * TILE + local / TILE;
        const int64_t i = (int64_t)A.tiles[2 * t + 1] * TILE + local % TILE;
        const int64_t r0 = j * k, c0 = i * k;
        // centre beds before the sort (wadi2d/tables/core.py:267-279)
        double cx, cy;
        {
            double col_a = INFINITY, col_b = INFINITY, row_a = INFINITY, row_b = INFINITY;
            const int ma = (k % 2) ? k / 2 : k / 2 - 1, mb = k / 2;
            for (int a = 0; a < k; ++a) {
                const double za = zpix(A, r0 + a, c0 + ma), zb = zpix(A, r0 + a, c0 + mb);
                col_a = za < col_a ? za : col_a;
                col_b = zb < col_b ? zb : col_b;
                const double ya = zpix(A, r0 + ma, c0 + a), yb = zpix(A, r0 + mb, c0 + a);
                row_a = ya < row_a ? ya : row_a;
                row_b = yb < row_b ? yb : row_b;
            }
            cx = (k % 2) ? col_b : 0.5 * (col_a + col_b);
            cy = (k % 2) ? row_b : 0.5 * (row_a + row_b);
        }
        for (int a = 0; a < k; ++a)
            for (int b = 0; b < k; ++b) p[a * k + b] = zpix(A, r0 + a, c0 + b);
        // ascending sort: insertion for small cells, heapsort beyond
        if (n <= 64) {
            for (int q = 1; q < n; ++q) {
                const double v = p[q];
                int s = q - 1;
                while (s >= 0 && p[s] > v) {
                    p[s + 1] = p[s];
                    --s;
                }
                p[s + 1] = v;
            }
        } else {
            for (int s = n / 2 - 1; s >= 0; --s) {
                int root = s;
                for (;;) {
                    int child = 2 * root + 1;
                    if (child >= n) break;
                    if (child + 1 < n && p[child] < p[child + 1]) ++child;
                    if (p[root] >= p[child]) break;
                    const double tmp = p[root];
                    p[root] = p[child];
                    p[child] = tmp;
                    root = child;
                }
            }
            for (int end = n - 1; end > 0; --end) {
                const double tmp = p[0];
                p[0] = p[end];
                p[end] = tmp;
                int root = 0;
                for (;;) {
                    int child = 2 * root + 1;
                    if (child >= end) break;
                    if (child + 1 < end && p[child] < p[child + 1]) ++child;
                    if (p[root] >= p[child]) break;
                    const double t2 = p[root];
                    p[root] = p[child];
                    p[child] = t2;
                    root = child;
                }
            }
        }
        // _cell_table, wadi2d/tables/core.py:16-41
        const double zmin = p[0];
        double sum = 0.0;
        for (int q = 0; q < n; ++q) {
            p[q] = p[q] - zmin;
            sum += p[q];
        }
        const double relmean = sum / (double)n;
        const double hc = p[n - 1] - relmean;
        float* tab = A.dtab + ((size_t)t * TILE2 + local) * rows;
        if (hc <= 1e-9) {
            for (int r = 0; r < rows; ++r) tab[r] = 0.0f;
            A.hc[(size_t)t * TILE2 + local] = 0.0f;
        } else {
            int m = 0;
            double cum = p[0];                 // sum of rel[0..m]
            double hb_m = (p[0] - cum) / (double)n;  // hbar_at[m]
            for (int r = 0; r < rows; ++r) {
                const double x = (double)r / (double)last;
                const double hb = hc * (x * x);
                while (m + 1 < n) {
                    const double cum1 = cum + p[m + 1];
                    const double hb1 = (p[m + 1] * (double)(m + 2) - cum1) / (double)n;
                    if (!(hb1 <= hb)) break;
                    m += 1;
                    cum = cum1;
                    hb_m = hb1;
                }
                const double v = p[m] + (hb - hb_m) * (double)n / (double)(m + 1);
                tab[r] = (float)(r == last ? p[n - 1] : v);
            }
            A.hc[(size_t)t * TILE2 + local] = (float)hc;
        }
        A.zmin[j * A.nx + i] = zmin;
        A.rel[j * A.nx + i] = relmean;
        // wadi2d/tables/builder.py:237, :248: centre beds over zmin, clamped at zero, NaN to zero
        double zx = cx - zmin, zy = cy - zmin;
        zx = isfinite(zx) ? (zx >= 0.0 ? zx : 0.0) : 0.0;
        zy = isfinite(zy) ? (zy >= 0.0 ? zy : 0.0) : 0.0;
        A.zcx[(size_t)t * TILE2 + local] = (float)zx;
        A.zcy[(size_t)t * TILE2 + local] = (float)zy;
    }
}

// ------------------------------------------------------------------ face tables (one thread per face)

// _face_table, wadi2d/tables/core.py:44-79, into tab[2 * rows] (FP64). prof is raised to the crest in place.
__device__ void face_table(double* prof, int m, double crest, double pixel, double n_inv, const double* weight,
                           double length, double e_lo, double e_hi, int rows, double* tab, double& zf_out,
                           double& top_out) {
    if (!isnan(crest))
        for (int q = 0; q < m; ++q) prof[q] = prof[q] >= crest ? prof[q] : crest;
    double zf = prof[0];
    for (int q = 1; q < m; ++q) zf = prof[q] < zf ? prof[q] : zf;
    double relmax = prof[0] - zf;
    for (int q = 1; q < m; ++q) {
        const double v = prof[q] - zf;
        relmax = v > relmax ? v : relmax;
    }
    const double lo = relmax <= e_hi ? relmax : e_hi;
    const double top = lo >= e_lo ? lo : e_lo;
    const int last = rows - 1;
    for (int r = 0; r < rows; ++r) {
        const double x = (double)r / (double)last;
        const double e = top * (x * x);
        double area = 0.0, conv = 0.0;
        for (int q = 0; q < m; ++q) {
            const double dep = e - (prof[q] - zf);
            if (dep > 0.0) {
                area += dep;
                const double cb = cbrt(dep);
                conv += weight[q] * dep * (cb * cb);
            }
        }
        tab[2 * r] = pixel * area * length;
        tab[2 * r + 1] = pow(pixel * n_inv * conv * length, 0.6);
    }
    zf_out = zf;
    top_out = top;
}

// _local_radius_conveyance, wadi2d/tables/core.py:82-179, on the line ext[0..n) held in the workspace (array 0);
// overwrites tab's conveyance column. W(a, i) is this thread's slot i of workspace array a.
struct Work {
    double* ws;
    int64_t stride;  // threads
    int64_t tid;
    int nmax;
    __device__ __forceinline__ double& operator()(int a, int i) const {
        return ws[((int64_t)a * (nmax + 1) + i) * stride + tid];
    }
};

enum { W_EXT = 0, W_D, W_PER, W_S0, W_S1, W_P0, W_P1, W_LO, W_HI };

__device__ void local_radius(const Work& W, int n, int i0, int i1, double zf, double top, double pixel,
                             double n_inv, const double* weight, double length, double beta, int rows, double* tab) {
    const double pix2 = pixel * pixel;
    const int last = rows - 1;
    for (int t = 0; t < n; ++t) {
        W(W_LO, t) = 0.0;
        W(W_HI, t) = 0.0;
    }
    W(W_S0, 0) = W(W_S1, 0) = W(W_P0, 0) = W(W_P1, 0) = 0.0;
    for (int r = 0; r < rows; ++r) {
        const double x = (double)r / (double)last;
        const double level = zf + top * (x * x);
        for (int t = 0; t < n; ++t) {
            const double dep = level - W(W_EXT, t);
            W(W_D, t) = dep > 0.0 ? dep : 0.0;
            W(W_PER, t) = 0.0;
        }
        if (W(W_D, 0) > 0.0) W(W_PER, 0) += 0.5 * pixel;
        if (W(W_D, n - 1) > 0.0) W(W_PER, n - 1) += 0.5 * pixel;
        for (int t = 0; t < n - 1; ++t) {
            const double da = W(W_D, t), db = W(W_D, t + 1);
            const bool wa = da > 0.0, wb = db > 0.0;
            if (!(wa || wb)) continue;
            const double rise = W(W_EXT, t + 1) - W(W_EXT, t);
            const double seg = sqrt(pix2 + rise * rise);
            if (wa && wb) {
                W(W_PER, t) += 0.5 * seg;
                W(W_PER, t + 1) += 0.5 * seg;
            } else if (wa) {
                if (rise > 0.0) {
                    const double f = da / rise;
                    W(W_PER, t) += (f <= 1.0 ? f : 1.0) * seg;
                } else {
                    W(W_PER, t) += 0.5 * pixel;
                }
            } else if (-rise > 0.0) {
                const double f = db / -rise;
                W(W_PER, t + 1) += (f <= 1.0 ? f : 1.0) * seg;
            } else {
                W(W_PER, t + 1) += 0.5 * pixel;
            }
        }
        int start = -1;
        for (int t = 0; t < n; ++t) {
            if (W(W_D, t) > 0.0) {
                if (start < 0) start = t;
                W(W_LO, t) = (double)start;
            } else {
                start = -1;
            }
        }
        int end = -1;
        for (int t = n - 1; t >= 0; --t) {
            if (W(W_D, t) > 0.0) {
                if (end < 0) end = t;
                W(W_HI, t) = (double)end;
            } else {
                end = -1;
            }
        }
        for (int t = 0; t < n; ++t) {
            const double d = W(W_D, t), per = W(W_PER, t);
            W(W_S0, t + 1) = W(W_S0, t) + d;
            W(W_S1, t + 1) = W(W_S1, t) + (double)t * d;
            W(W_P0, t + 1) = W(W_P0, t) + per;
            W(W_P1, t + 1) = W(W_P1, t) + (double)t * per;
        }
        double conv = 0.0;
        for (int i = i0; i < i1; ++i) {
            const double di = W(W_D, i);
            if (di <= 0.0) continue;
            double w = beta * di / pixel;
            if (w < 1e-9) w = 1e-9;
            int lo = (int)ceil((double)i - w);
            const int rlo = (int)W(W_LO, i);
            lo = rlo > lo ? rlo : lo;
            int hi = (int)floor((double)i + w);
            const int rhi = (int)W(W_HI, i);
            hi = rhi < hi ? rhi : hi;
            const double fi = (double)i;
            double a_sum = (1.0 - fi / w) * (W(W_S0, i + 1) - W(W_S0, lo)) + (W(W_S1, i + 1) - W(W_S1, lo)) / w;
            a_sum += (1.0 + fi / w) * (W(W_S0, hi + 1) - W(W_S0, i + 1)) - (W(W_S1, hi + 1) - W(W_S1, i + 1)) / w;
            double p_sum = (1.0 - fi / w) * (W(W_P0, i + 1) - W(W_P0, lo)) + (W(W_P1, i + 1) - W(W_P1, lo)) / w;
            p_sum += (1.0 + fi / w) * (W(W_P0, hi + 1) - W(W_P0, i + 1)) - (W(W_P1, hi + 1) - W(W_P1, i + 1)) / w;
            const double radius = p_sum > 0.0 ? pixel * a_sum / p_sum : di;
            const double cb = cbrt(radius);
            conv += weight[i - i0] * di * (cb * cb);
        }
        tab[2 * r + 1] = pow(pixel * n_inv * conv * length, 0.6);
    }
}

constexpr int KMAX = 32;
constexpr int64_t FACE_SMEM_BYTES = 200 * 1024;  // the shared workspace a CTA of the face-table kernel may take
constexpr int ROWS_MAX = 64;

// SMEM: the local radius's workspace in this CTA's shared memory (interleaved across its threads as the global one is
// across the grid's), else in the caller's device workspace. The arithmetic is the same either way.
template <bool SMEM>
__global__ void __launch_bounds__(128) face_tables_kernel(TableArgs A) {
    extern __shared__ double sws[];
    const int64_t nface = (int64_t)(A.ntiles - 1) * TILE2 * 2;
    const int k = A.k, rows = A.rows;
    double prof[KMAX], weight[KMAX], tab[2 * ROWS_MAX];
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const Work W = SMEM ? Work{sws, (int64_t)blockDim.x, (int64_t)threadIdx.x, A.nmax} : Work{A.ws, A.ws_threads, tid, A.nmax};
    for (int64_t f = tid; f < nface; f += (int64_t)gridDim.x * blockDim.x) {
        const int axis = (int)(f & 1);
        const int64_t c = f >> 1;
        const int t = (int)(c / TILE2) + 1;
        const int local = (int)(c % TILE2);
        const int64_t j = (int64_t)A.tiles[2 * t] * TILE + local / TILE;
        const int64_t i = (int64_t)A.tiles[2 * t + 1] * TILE + local % TILE;
        const int64_t r0 = j * k, c0 = i * k;
        const int64_t g = j * A.nx + i;
        const double nm = A.nman[g];
        // the higher of the two pixels meeting along the face, and its lining (wadi2d/tables/core.py:249-264)
        for (int q = 0; q < k; ++q) {
            int64_t nr, nc, fr, fc;
            if (axis == 0) {
                nr = r0 + q, nc = c0, fr = r0 + q, fc = c0 - 1;
            } else {
                nr = r0, nc = c0 + q, fr = r0 - 1, fc = c0 + q;
            }
            const double near = zpix(A, nr, nc), far = zpix(A, fr, fc);
            prof[q] = far >= near ? far : near;
            weight[q] = A.npix ? lined(far > near ? npix_at(A, fr, fc) : npix_at(A, nr, nc), nm) : 1.0;
        }
        const double crest = axis == 0 ? A.xcrest[g] : A.ycrest[g];
        const double length = axis == 0 ? A.xlen[g] : A.ylen[g];
        double zf, top;
        face_table(prof, k, crest, A.pixel, 1.0 / nm, weight, length, A.e_lo, A.e_hi, rows, tab, zf, top);
        if (A.local && isnan(crest)) {
            // wadi2d/tables/core.py:324-351: the face's line reaches margin pixels past both ends
            const int nfull = k + 2 * A.margin;
            double hi = -INFINITY;
            for (int s = 0; s < nfull; ++s) {
                double x0, x1;
                if (axis == 0) {
                    x0 = zpix(A, r0 + s - A.margin, c0 - 1);
                    x1 = zpix(A, r0 + s - A.margin, c0);
                } else {
                    x0 = zpix(A, r0 - 1, c0 + s - A.margin);
                    x1 = zpix(A, r0, c0 + s - A.margin);
                }
                const double v = x0 >= x1 ? x0 : x1;
                W(W_EXT, s) = v;
                hi = v > hi ? v : hi;
            }
            // _raise_top and window_top, wadi2d/tables/core.py:354-371
            const double relw = hi - zf;
            const double cap = relw <= A.e_hi ? relw : A.e_hi;
            const double wtop = top >= cap ? top : cap;
            if (wtop > top) {
                for (int q = 0; q < k; ++q) prof[q] = W(W_EXT, A.margin + q);
                face_table(prof, k, NAN, A.pixel, 1.0 / nm, weight, length, wtop, A.e_hi, rows, tab, zf, top);
            }
            int e = (int)ceil(A.beta * top / A.pixel);
            e = e > A.margin ? A.margin : e;
            // the conveyance line is full[margin - e : margin + k + e]: shift it to the front of the workspace
            const int off = A.margin - e;
            const int nn = k + 2 * e;
            if (off > 0)
                for (int s = 0; s < nn; ++s) W(W_EXT, s) = W(W_EXT, s + off);
            local_radius(W, nn, e, e + k, zf, top, A.pixel, 1.0 / nm, weight, length, A.beta, rows, tab);
        }
        float* out = (axis == 0 ? A.ftabx : A.ftaby) + ((size_t)t * TILE2 + local) * rows * 2;
        for (int r = 0; r < 2 * rows; ++r) out[r] = (float)tab[r];
        (axis == 0 ? A.efx : A.efy)[(size_t)t * TILE2 + local] = (float)top;
        (axis == 0 ? A.zfx : A.zfy)[g] = zf;
    }
}

// ------------------------------------------------------------------ inverts, closed faces, crests (per face)

// _faces, wadi2d/tables/builder.py:290-308; the neighbour is (j, i-1) for x faces and (j-1, i) for y faces, with
// np.roll's wrap at the grid edge.
__global__ void close_faces_kernel(TableArgs A) {
    const int64_t nface = (int64_t)(A.ntiles - 1) * TILE2 * 2;
    for (int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; f < nface; f += (int64_t)gridDim.x * blockDim.x) {
        const int axis = (int)(f & 1);
        const int64_t c = f >> 1;
        const int t = (int)(c / TILE2) + 1;
        const int local = (int)(c % TILE2);
        const int64_t j = (int64_t)A.tiles[2 * t] * TILE + local / TILE;
        const int64_t i = (int64_t)A.tiles[2 * t + 1] * TILE + local % TILE;
        const int64_t g = j * A.nx + i;
        const int64_t gn = axis == 0 ? j * A.nx + (i == 0 ? A.nx - 1 : i - 1) : (j == 0 ? A.ny - 1 : j - 1) * A.nx + i;
        const double zf = axis == 0 ? A.zfx[g] : A.zfy[g];
        const uint8_t* wall = axis == 0 ? A.xwall : A.ywall;
        const bool open = A.mask[g] && A.mask[gn] && !(wall && wall[g]);
        const double zmin = A.zmin[g], zmin_n = A.zmin[gn];
        const double zbar = zmin + A.rel[g], zbar_n = zmin_n + A.rel[gn];
        const double fl = open ? zf - zmin_n : 1.0e9;
        const double fr = open ? zf - zmin : 1.0e9;
        const double gl = open ? zf - zbar_n : 0.0;
        const double gr = open ? zf - zbar : 0.0;
        const bool natural = open && (gl > A.tol) && (gr > A.tol);
        const double given = axis == 0 ? A.xc[g] : A.yc[g];
        double cw = given != 0.0 ? given : (natural ? 1.7046 : 0.0);
        cw = open ? cw : 0.0;
        const size_t o = (size_t)t * TILE2 + local;
        (axis == 0 ? A.flx : A.fly)[o] = (float)fl;
        (axis == 0 ? A.frx : A.fry)[o] = (float)fr;
        (axis == 0 ? A.glx : A.gly)[o] = (float)gl;
        (axis == 0 ? A.grx : A.gry)[o] = (float)gr;
        (axis == 0 ? A.cwx : A.cwy)[o] = (float)cw;
    }
}

}  // namespace w2b

using namespace w2b;

extern "C" {

int64_t w2b_table_workspace_doubles(int32_t nmax, int64_t threads) { return 9 * (int64_t)(nmax + 1) * threads; }

int32_t w2b_build_tables(const W2BTableIn* in, const W2BTableOut* out, void* stream) {
    if (!in || !out || !in->z || !in->nman || !in->mask || !in->tiles || in->k < 1 || in->k > KMAX || in->rows < 4 ||
        in->rows > ROWS_MAX || in->ntiles < 1 || in->ny % TILE || in->nx % TILE || in->zh < 1 || in->zw < 1)
        return W2B_EINVAL;
    if (in->local && (!out->ws || out->ws_threads < 1)) return W2B_EINVAL;
    if (in->local && (in->margin < 0 || in->margin > W2B_TABLE_MARGIN_MAX)) return W2B_EINVAL;
    TableArgs A;
    A.z = in->z;
    A.zh = in->zh;
    A.zw = in->zw;
    A.roff = in->row_offset;
    A.coff = in->col_offset;
    A.npix = in->npix;
    A.nman = in->nman;
    A.xcrest = in->xcrest;
    A.xlen = in->xlen;
    A.xc = in->xc;
    A.ycrest = in->ycrest;
    A.ylen = in->ylen;
    A.yc = in->yc;
    A.xwall = in->xwall;
    A.ywall = in->ywall;
    A.mask = in->mask;
    A.tiles = in->tiles;
    A.ntiles = in->ntiles;
    A.ny = in->ny;
    A.nx = in->nx;
    A.k = in->k;
    A.rows = in->rows;
    A.local = in->local;
    A.margin = in->local ? in->margin : 0;
    A.nmax = in->k + 2 * A.margin;
    A.pixel = in->pixel;
    A.e_lo = in->face_depth_min;
    A.e_hi = in->face_depth_max;
    A.beta = in->beta;
    A.tol = in->crest_tolerance;
    A.hc = out->hc;
    A.dtab = out->dtab;
    A.efx = out->efx;
    A.efy = out->efy;
    A.ftabx = out->ftabx;
    A.ftaby = out->ftaby;
    A.zcx = out->zcx;
    A.zcy = out->zcy;
    A.flx = out->flx;
    A.frx = out->frx;
    A.glx = out->glx;
    A.grx = out->grx;
    A.cwx = out->cwx;
    A.fly = out->fly;
    A.fry = out->fry;
    A.gly = out->gly;
    A.gry = out->gry;
    A.cwy = out->cwy;
    A.zmin = out->zmin;
    A.rel = out->rel;
    A.zfx = out->zfx;
    A.zfy = out->zfy;
    A.ws = out->ws;
    A.ws_threads = out->ws_threads;
    if (in->local && out->ws_threads % 128) return W2B_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    const int n = in->k * in->k;
    const int cblocks = 148 * 8;
    if (n <= 64)
        cell_tables_kernel<64><<<cblocks, 128, 0, s>>>(A);
    else if (n <= 256)
        cell_tables_kernel<256><<<cblocks, 128, 0, s>>>(A);
    else
        cell_tables_kernel<1024><<<cblocks, 128, 0, s>>>(A);
    // the local radius's workspace: in shared memory when a CTA of at least one thread fits it (a face line of up to
    // about 2,800 pixels), else in the caller's workspace
    const int64_t per_thread = 9 * (int64_t)(A.nmax + 1) * (int64_t)sizeof(double);
    const int64_t smem_threads = in->local ? FACE_SMEM_BYTES / per_thread : 0;
    if (in->local && smem_threads >= 1) {
        const int threads = smem_threads > 128 ? 128 : (int)smem_threads;
        const size_t bytes = (size_t)threads * (size_t)per_thread;
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (cudaFuncSetAttribute(face_tables_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) !=
            cudaSuccess) {
            fprintf(stderr, "libwadi_b200: w2b_build_tables: shared workspace: %s\n",
                    cudaGetErrorString(cudaGetLastError()));
            return W2B_ECUDA;
        }
        // as many CTAs a SM as their workspaces allow: short face lines leave room for several
        int occ = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, face_tables_kernel<true>, threads, bytes) !=
                cudaSuccess ||
            occ < 1)
            occ = 1;
        face_tables_kernel<true><<<sms * occ, threads, bytes, s>>>(A);
    } else {
        const int64_t fthreads = in->local ? out->ws_threads : (int64_t)148 * 8 * 128;
        face_tables_kernel<false><<<(unsigned)(fthreads / 128), 128, 0, s>>>(A);
    }
    close_faces_kernel<<<148 * 8, 256, 0, s>>>(A);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "libwadi_b200: w2b_build_tables: %s\n", cudaGetErrorString(e));
        return W2B_ECUDA;
    }
    return W2B_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ the table build without allocation

// Scratch of w2b_build_tables_noalloc: 32 MiB of file-scope device memory. Every GPU on which a process loads this
// library holds it until the process exits, whether the entry point is called or not.
constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)32 << 20;
static __device__ __align__(256) double noalloc_scratch[NOALLOC_SCRATCH_BYTES / sizeof(double)];

// The array's device address, looked up once per device with that device current and kept for the life of the
// process (a cudaDeviceReset makes it stale). In host code the name noalloc_scratch is a host-side stand-in, not a
// device address: a kernel given it would fault or read the wrong memory, so only this address is ever passed on.
static std::mutex noalloc_mutex;
static void* noalloc_address[256];

static int noalloc_scratch_address(void** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return W2B_ECUDA;
    std::lock_guard<std::mutex> lock(noalloc_mutex);
    if (!noalloc_address[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, noalloc_scratch);
        if (e != cudaSuccess || !p) {
            fprintf(stderr, "libwadi_b200: w2b_build_tables_noalloc: cudaGetSymbolAddress: %s\n",
                    cudaGetErrorString(e));
            return W2B_ECUDA;
        }
        noalloc_address[dev] = p;
    }
    *out = noalloc_address[dev];
    return W2B_OK;
}

extern "C" int32_t w2b_build_tables_noalloc(const W2BTableIn* in, const W2BTableOut* out, void* stream) {
    if (!in || !out) return W2B_EINVAL;
    if (in->local && (in->margin < 0 || in->margin > W2B_TABLE_MARGIN_MAX)) return W2B_EINVAL;
    W2BTableOut o = *out;
    o.ws = nullptr;
    o.ws_threads = 0;
    if (in->local) {
        const int64_t per_thread = 9 * ((int64_t)in->k + 2 * (int64_t)in->margin + 1) * (int64_t)sizeof(double);
        const int64_t threads = (int64_t)(NOALLOC_SCRATCH_BYTES / (size_t)per_thread) / 128 * 128;
        if (threads < 128) {
            fprintf(stderr,
                    "libwadi_b200: w2b_build_tables_noalloc: face lines of %d pixels need %lld bytes of scratch for "
                    "128 threads; the static scratch holds %zu (at most %lld pixels a line)\n",
                    in->k + 2 * in->margin, (long long)(per_thread * 128), NOALLOC_SCRATCH_BYTES,
                    (long long)(NOALLOC_SCRATCH_BYTES / (128 * 9 * sizeof(double)) - 1));
            return W2B_EINVAL;
        }
        void* ws = nullptr;
        const int st = noalloc_scratch_address(&ws);
        if (st != W2B_OK) return st;
        o.ws = static_cast<double*>(ws);
        o.ws_threads = threads;
    }
    return w2b_build_tables(in, &o, stream);
}
