// Shared device definitions of libwadi_b200: layout constants, the control block, the argument records, and the
// float32 helpers of the step. The helpers restate wadi2d/solver/gpu/kernels/common.cuh:22-96 (= the Numba twin
// wadi2d/solver/cpu/kernels.py:19-83) in the same statement order; the library is compiled with -fmad=false and
// IEEE division and square root, so with identical inputs each helper returns the reference CPU twin's bits.
#pragma once

#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include "wadi_b200.h"

namespace w2b {

constexpr int TILE = 32;
constexpr int TILE2 = TILE * TILE;
constexpr int GY = 4;   // guard rows above and below the padded grid in the native layout
constexpr int GX = 32;  // guard columns left and right: keeps every tile row 128-byte aligned
constexpr int SLEEP_CHECKS = 2;  // wadi2d/solver/stepper.py:12

// Device control block, W2B_CTL_BYTES long: what the step kernels share across runs. Each run's own clock and step
// settings live in the run table (RunTab); a single run is run 0 of a table of one.
struct Ctl {
    int32_t nact;       // active tiles (all runs)
    int32_t nwork;      // entries of the work list the face and update passes take
    int32_t prune;      // a run stopped stepping: the work list is to be rebuilt
    uint32_t any;       // ANY_* bits: OR over the runs of this step's flags
    int32_t nwoken;     // tiles the last rebuild woke
    int32_t status;     // a failure no single run owns (W2B_ETIMEOUT)
    int32_t nruns;
    int32_t dt_every, active_every, adaptive, max_every;
    float arrive, deep;
    double cfl, wave_floor, dt_max, dt_min;
    // 1 while the momentum arrays hold the face momenta (set at creation and by w2b_sync_momentum), 0 once a face pass
    // has stepped: the face pass then forms each face's momentum from the state instead of reading it (the momentum
    // after a step is abar * u with abar from the mean depths the step started from, which are still the other half
    // of the ping-pong pair). Last member: the device loop's settings overwrite the block up to it.
    int32_t m_stored;
};
static_assert(sizeof(Ctl) <= W2B_CTL_BYTES, "control block too large");

constexpr uint32_t ANY_RUN = 1u, ANY_WAVE = 2u, ANY_ACT = 4u, ANY_MAX = 8u;
// per-run flags of this step
constexpr int32_t F_RUN = 1, F_WAVE = 2, F_WET = 4, F_MAX = 8, F_ACT = 16;

// Per-run state, one entry a run (wadi2d/solver/stepper.py:24-47 for each run of a batch).
struct RunTab {
    double *t, *dt, *t_end, *dt_step, *dt_tally;
    long long *nsteps, *steps_run, *max_steps;
    float *dtf, *max_time, *dx;
    int32_t *flags, *refresh_due, *status;
    uint32_t* wave_bits;  // max wave speed of the run's tiles, as float bits (waves are never negative)
    int32_t* parity;      // the run's current half of the ping-pong pairs
    float* wave_last;     // the wave maximum of the run's last refresh step (what the clock reports)
};

// Whether run r takes another step (the loop test of wadi2d/solver/stepper.py:106, plus the batch's step limit).
__device__ __forceinline__ bool live_run(const RunTab& R, int r, const Ctl* ctl) {
    return ctl->status == 0 && R.status[r] == 0 && R.t[r] < R.t_end[r] - 1e-9 && R.steps_run[r] < R.max_steps[r];
}

// Layout of a run table of nruns entries in one device block: each array 256-byte aligned.
__host__ __device__ inline size_t run_table_bytes(int nruns) {
    const size_t a = ((size_t)nruns * 8 + 255) / 256 * 256, b = ((size_t)nruns * 4 + 255) / 256 * 256;
    return 8 * a + 9 * b;
}

__host__ __device__ inline RunTab run_table(void* base, int nruns) {
    const size_t a = ((size_t)nruns * 8 + 255) / 256 * 256, b = ((size_t)nruns * 4 + 255) / 256 * 256;
    char* p = static_cast<char*>(base);
    RunTab R;
    R.t = reinterpret_cast<double*>(p);
    R.dt = reinterpret_cast<double*>(p + a);
    R.t_end = reinterpret_cast<double*>(p + 2 * a);
    R.dt_step = reinterpret_cast<double*>(p + 3 * a);
    R.dt_tally = reinterpret_cast<double*>(p + 4 * a);
    R.nsteps = reinterpret_cast<long long*>(p + 5 * a);
    R.steps_run = reinterpret_cast<long long*>(p + 6 * a);
    R.max_steps = reinterpret_cast<long long*>(p + 7 * a);
    char* q = p + 8 * a;
    R.dtf = reinterpret_cast<float*>(q);
    R.max_time = reinterpret_cast<float*>(q + b);
    R.dx = reinterpret_cast<float*>(q + 2 * b);
    R.flags = reinterpret_cast<int32_t*>(q + 3 * b);
    R.refresh_due = reinterpret_cast<int32_t*>(q + 4 * b);
    R.status = reinterpret_cast<int32_t*>(q + 5 * b);
    R.wave_bits = reinterpret_cast<uint32_t*>(q + 6 * b);
    R.parity = reinterpret_cast<int32_t*>(q + 7 * b);
    R.wave_last = reinterpret_cast<float*>(q + 8 * b);
    return R;
}

// Everything a step kernel reads, with the ping-pong halves resolved for one parity.
struct StepArgs {
    W2BParams P;
    int32_t rows, px, ntiles, nty, ntx;
    // state, native; ping-pong pairs by half: a run's current half is R.parity[run], the other is the next
    float* hh[2];     // mean depth
    float* uu[2][2];  // face velocities [axis x, y][half]
    float* mm[2][2];  // face momenta [axis][half]
    float* __restrict__ d;
    float* __restrict__ q[2];   // qx, qy: scaled discharges
    float* __restrict__ q1[2];  // qx1, qy1: unscaled, from the face pass
    float* __restrict__ res;
    const float* __restrict__ src;
    float* __restrict__ om;
    const float* __restrict__ zc[2];
    // static, tile layout
    const float* __restrict__ hc;
    const float* __restrict__ fl[2];
    const float* __restrict__ fr[2];
    const float* __restrict__ gl[2];
    const float* __restrict__ gr[2];
    const float* __restrict__ ef[2];
    const float* __restrict__ cw[2];
    const float2* __restrict__ dtab2;
    const float4* __restrict__ ftab4[2];
    const int32_t* __restrict__ table_tile;  // the static and table tile of each tile, or null: its own
    const int32_t* __restrict__ tiles;
    const int32_t* __restrict__ tile_of;
    const int32_t* __restrict__ nbr;
    int32_t* __restrict__ active;
    float* __restrict__ wave;
    int32_t* __restrict__ wet;
    int32_t* __restrict__ keep;
    int32_t* __restrict__ idle;
    int32_t* __restrict__ is_act;
    int32_t* __restrict__ woken;
    const int32_t* __restrict__ list;  // the tiles the face and update passes take (ctl->nwork of them)
    int32_t* __restrict__ work;        // the device loop's work list
    int32_t* __restrict__ scratch;
    float* __restrict__ env[5];
    const uint32_t* __restrict__ bmark;
    // boundary cells and tally faces
    int32_t nb;
    const int32_t* __restrict__ bcell;
    const int32_t* __restrict__ bref;
    const int32_t* __restrict__ bkind;
    const float* __restrict__ bd0;
    const float* __restrict__ bh0;
    int32_t ntally;
    const int32_t* __restrict__ tface;
    const int32_t* __restrict__ taxis;
    const float* __restrict__ tsign;
    double* __restrict__ ttotal;
    // design lines: line l's faces are lface[lstart[l] .. lstart[l + 1]); discharge now, its peak |Q| and the time
    int32_t nlines;
    const int32_t* __restrict__ lstart;
    const int32_t* __restrict__ lface;
    const int32_t* __restrict__ laxis;
    const float* __restrict__ lsign;
    double* __restrict__ lq;
    double* __restrict__ lpeak;
    double* __restrict__ ltime;
    Ctl* ctl;
    // runs: the run of each tile, and the run table
    const int32_t* __restrict__ tile_run;
    RunTab R;
    // the update pass's level cache: each cell's last level pair and its row (0xff: none), tile layout
    float2* __restrict__ lpair;
    uint8_t* __restrict__ lrow;
    int32_t nruns;
};

// Tensor maps of the NATIVE state arrays for the face pass's TMA boxes: 40 x 36 floats (the tile, two cells of halo
// north and south, four west and east so that the box's first column stays 16-byte aligned), and 32 x 32 for the
// momenta, which the face pass reads at own faces only. Ping-pong pairs have one map a half.
// The strip forms of the face pass (strips of H rows of a tile): 40 x (H + 4) boxes, and 32 x H for the momenta.
struct StripMaps {
    CUtensorMap d, h[2], u[2], v[2], qx, qy, zcx, zcy, mx[2], my[2];
};
struct TMaps {
    CUtensorMap d, h[2], u[2], v[2], qx, qy, om, zcx, zcy, mx[2], my[2];
    CUtensorMap qx1, qy1;  // 40 x 36 boxes for the update pass
    CUtensorMap res, src;  // 32 x 32 boxes
    StripMaps s16, s8;     // strips of 16 and of 8 rows
};

// ------------------------------------------------------------------ float32 helpers

// x > m^3 for a midpoint m between two adjacent floats, decided exactly. m has a 25-bit significand, so m * m is
// exact in double and m^3 = p + e exactly with p = fl(m^2 m) and e = fma(m^2, m, -p); x lies within a factor two of
// p, so x - p is exact (Sterbenz) and x > m^3 exactly when x - p > e.
__device__ __forceinline__ bool cube_above(double m, float x) {
    const double m2 = m * m;
    const double p = m2 * m;
    const double e = fma(m2, m, -p);
    return (double)x - p > e;
}

// The float nearest the cube root of x, decided exactly in double: cbrtf gives a float within one ulp; of it and its
// two neighbours the answer is decided by comparing x with the cubes of the two midpoints (cube_above). The path for
// the ends of the float range, and for the rare inputs whose FP32 decision in cbrt32 is too close to call.
static __device__ __noinline__ float cbrt32_exact(float x) {
    if (!(x > 0.0f) || x > 3.0e38f) return (float)cbrt((double)x);  // zero, negative, NaN, huge: the double path
    const float y = cbrtf(x);
    const float yu = __int_as_float(__float_as_int(y) + 1);
    const float yd = __int_as_float(__float_as_int(y) - 1);
    if (cube_above(0.5 * ((double)y + (double)yu), x)) return yu;
    if (!cube_above(0.5 * ((double)yd + (double)y), x)) return yd;
    return y;
}

// The hardware's base-2 logarithm, exponential and reciprocal estimates (PTX lg2.approx, ex2.approx, rcp.approx; the
// inputs here are positive normal floats).
__device__ __forceinline__ float lg2_approx(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// The float nearest the cube root of x. Numba's float32 cbrt is float(cbrt(double(x))), the cube root rounded once to
// double and once to float; this returns the correctly rounded float, which is the same number whenever the double
// root is within the distance of cbrt(x) from the nearest float midpoint (w2b_selftest_cbrt compares the two over
// every positive float). Method, in FP32 for 2^-96 <= x <= 2^96:
//  - y0 = 2^(log2(x) / 3) from the hardware estimates is within 2^-19 of the root t; one Newton step,
//    y = y0 - (y0^3 - x) / (3 y0^2), with y0^3 - x formed from an error-free square, is within half an ulp plus
//    2^-36 t of t, so the answer is y or its neighbour on the side of t;
//  - d = x - y^3 to within 2^-45 x: y^2 = q + qe and q y = c + ce exactly (FMA error-free products), x - c exactly
//    (Sterbenz), the tail qe y rounded once; its sign gives the side of t;
//  - with s the signed half-ulp step to that side's midpoint m = y + s, x - m^3 = d - (3 y^2 s + 3 y s^2 + s^3), the
//    roundings below 2^-44 x in all; a value beyond 2^-42 x has a certain sign and picks the answer, a value inside
//    it (about one input in 2^17) and x outside the range go to cbrt32_exact.
__device__ __forceinline__ float cbrt32(float x) {
    if (!(x >= 0x1p-96f && x <= 0x1p96f)) return cbrt32_exact(x);
    const float y0 = ex2_approx(lg2_approx(x) * 0.333333343f);
    const float p = y0 * y0;
    const float pe = fmaf(y0, y0, -p);
    const float r = fmaf(p, y0, -x) + pe * y0;  // y0^3 - x
    const float y = fmaf(-r, rcp_approx(3.0f * p), y0);
    const float q = y * y;
    const float qe = fmaf(y, y, -q);
    const float c = q * y;
    const float ce = fmaf(q, y, -c);
    const float d = ((x - c) - ce) - qe * y;  // x - y^3
    const int bits = __float_as_int(y);
    const float nb = __int_as_float(d >= 0.0f ? bits + 1 : bits - 1);
    const float st = 0.5f * (nb - y);  // exact: half the gap to the neighbour, signed
    const float z = d - (3.0f * q * st + 3.0f * y * st * st);
    if (fabsf(z) <= x * 0x1p-42f) return cbrt32_exact(x);
    return (z > 0.0f) == (d >= 0.0f) ? nb : y;
}
// The face pass's division, square root and cube root. The library's default build is the reference's arithmetic:
// IEEE division and square root (it is compiled with -prec-div=true -prec-sqrt=true -fmad=false) and the correctly
// rounded cube root, so these are a / b, sqrtf and cbrt32. The step's second build (W2B_FAST, compiled with FMA
// contraction; selected per handle by W2BParams.arith) uses the hardware's approximations where the face pass spends
// its instructions:
//  - division as div.approx.ftz (the numerator times rcp.approx, within 2 ulp while the denominator's magnitude lies
//    in [2^-126, 2^126]: every denominator of the face pass is a depth, area, width, cell size or clamp of them,
//    bounded below by 1e-30 or by e_wet);
//  - sqrt.approx.ftz (within about 1 ulp);
//  - the cube root of x >= 0 from the hardware log2 and exp2 estimates (within about 2^-18 relative) refined by one
//    Newton step, y - (y^3 - x) / (3 y^2), which squares that error away: within a few ulp. x = 0, and x so small that
//    the estimate is 0, give 0.
// The .ftz forms take a subnormal operand or result as zero, so they need no rescaling around the hardware estimate:
// a quotient or root that would have been subnormal (below 2^-126, about 1.2e-38) reads as 0, an absolute change
// smaller than that.
__device__ __forceinline__ float div_approx(float a, float b) {
    float y;
    asm("div.approx.ftz.f32 %0, %1, %2;" : "=f"(y) : "f"(a), "f"(b));
    return y;
}
__device__ __forceinline__ float sqrt_approx(float x) {
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float cbrt_fast(float x) {
    const float y0 = ex2_approx(lg2_approx(x) * 0.333333343f);
    const float p = y0 * y0;
    const float y = fmaf(-fmaf(p, y0, -x), rcp_approx(3.0f * p), y0);
    return y0 > 0.0f ? y : y0;
}
// Python max/min on two ordered floats (the first argument wins a tie).
__device__ __forceinline__ float fmax32(float a, float b) { return a >= b ? a : b; }
__device__ __forceinline__ float fmin32(float a, float b) { return a <= b ? a : b; }

#ifdef W2B_FAST
__device__ __forceinline__ float qdiv(float a, float b) { return div_approx(a, b); }
__device__ __forceinline__ float qsqrt(float x) { return sqrt_approx(x); }
__device__ __forceinline__ float qcbrt(float x) { return cbrt_fast(x); }
// the hardware max and min, one instruction each: the same as fmax32 / fmin32 for ordered operands but for the sign of
// a zero tie, and they return the other operand where one is NaN
__device__ __forceinline__ float qmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ float qmin(float a, float b) { return fminf(a, b); }
#else
__device__ __forceinline__ float qdiv(float a, float b) { return a / b; }
__device__ __forceinline__ float qsqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ float qcbrt(float x) { return cbrt32(x); }
__device__ __forceinline__ float qmax(float a, float b) { return fmax32(a, b); }
__device__ __forceinline__ float qmin(float a, float b) { return fmin32(a, b); }
#endif

__device__ __forceinline__ float minmod(float a, float b) {
    if (a * b <= 0.0f) return 0.0f;
    return fabsf(a) < fabsf(b) ? a : b;
}

// Velocity at a cell centre from its upwind face uc, with a limited second-order correction (common.cuh:30-34).
__device__ __forceinline__ float ustar(float uc, float uup, float udown, int second) {
    if (!second) return uc;
    return uc + 0.5f * minmod(uc - uup, udown - uc);
}

__device__ __forceinline__ float gated(float neighbour, float own, int mirror) {
    return (mirror && neighbour == 0.0f) ? own : neighbour;
}

__device__ __forceinline__ bool not_finite(float v) { return (__float_as_int(v) & 0x7f800000) == 0x7f800000; }

// Row index of a quadratic table, clamped to [0, last - 1] so that no input can read outside the table.
__device__ __forceinline__ int row_of(float s, int last) {
    int r = (int)s;
    r = r < 0 ? 0 : r;
    return r > last - 1 ? last - 1 : r;
}

// Level above zmin from mean depth, wadi2d/solver/gpu/kernels/common.cuh:39-47. pair(r) = (tab[r], tab[r + 1]).
__device__ __forceinline__ float cell_level(float hb, float hc, const float2* __restrict__ pairs, int rows,
                                            int fp64) {
    if (hc <= 0.0f) return hb;
    const int last = rows - 1;
    if (hb >= hc) {
        const float2 p = __ldg(pairs + (size_t)(last - 1) * TILE2);
        return p.y + (hb - hc);
    }
    const float s = sqrtf(hb / hc) * (float)last;
    const int r = row_of(s, last);
    const float2 p = __ldg(pairs + (size_t)r * TILE2);
    if (fp64 && r == 0) {
        // near-dry bottom interval: the row coordinate and the interpolation in FP64
        const double sd = sqrt((double)hb / (double)hc) * (double)last;
        return (float)((double)p.x + sd * ((double)p.y - (double)p.x));
    }
    return p.x + (s - (float)r) * (p.y - p.x);
}

// Wet share of the cell plan, wadi2d/solver/gpu/kernels/common.cuh:49-57.
__device__ __forceinline__ float cell_plan(float hb, float hc, const float2* __restrict__ pairs, int rows) {
    if (hc <= 0.0f || hb >= hc) return 1.0f;
    const int last = rows - 1;
    const float s = sqrtf(hb / hc) * (float)last;
    const int r = row_of(s, last);
    const float m = (float)last;
    const float2 p = __ldg(pairs + (size_t)r * TILE2);
    return hc * (float)(2 * r + 1) / (m * m) / fmax32(p.y - p.x, 1e-12f);
}

// Area, conveyance^(3/5) and wet width at depth e over the face invert, wadi2d/solver/gpu/kernels/common.cuh:64-91
// (with the face pass's division and square root).
// quad(r) = (A_r, T_r, A_r+1, T_r+1).
__device__ __forceinline__ void face_lookup(float e, float top, const float4* __restrict__ quads, int rows, float& A,
                                            float& T, float& W) {
    const int last = rows - 1;
    const float m = (float)last;
    if (e >= top) {
        const float4 q = __ldg(quads + (size_t)(last - 1) * TILE2);
        const float a1 = q.z;
        const float a0 = q.x;
        const float c = qdiv(m - 1.0f, m);
        W = qdiv(a1 - a0, top * (1.0f - c * c));
        A = a1 + W * (e - top);
        T = q.w * qdiv(A, fmax32(a1, 1e-12f));
        return;
    }
    const float s = qsqrt(qdiv(e, top)) * m;
    const int r = row_of(s, last);
    const float c0 = qdiv((float)r, m);
    const float c1 = qdiv((float)(r + 1), m);
    const float e0 = c0 * c0 * top;
    const float de = (c1 * c1 - c0 * c0) * top;
    const float f = qdiv(e - e0, de);
    const float4 q = __ldg(quads + (size_t)r * TILE2);
    A = q.x + f * (q.z - q.x);
    T = q.y + f * (q.w - q.y);
    W = qdiv(q.z - q.x, de);
}

// The tile whose static arrays and tables tile t reads (runs of a batch on one catchment share one copy).
__device__ __forceinline__ int table_of(const StepArgs& A, int t) { return A.table_tile ? A.table_tile[t] : t; }

// The tile holding NATIVE index k, and the tile-layout index of k's cell.
__device__ __forceinline__ int tile_of_native(const StepArgs& A, int k) {
    const int j = k / A.px - GY;
    const int i = k - (j + GY) * A.px - GX;
    return A.tile_of[(j / TILE) * A.ntx + (i / TILE)];
}

__device__ __forceinline__ int fid_of_native(const StepArgs& A, int k) {
    const int j = k / A.px - GY;
    const int i = k - (j + GY) * A.px - GX;
    const int t = A.tile_of[(j / TILE) * A.ntx + (i / TILE)];
    return t * TILE2 + (j % TILE) * TILE + (i % TILE);
}

// The step arguments of a handle (for kernels of other translation units); false on a null handle.
bool handle_args(void* handle, StepArgs* out);

}  // namespace w2b
