/*
 * wadi_b200.h -- C-ABI of libwadi_b200.so, the B200 (sm_100a) form of Wadi2D's uniform-grid shallow-water step.
 *
 * The library drops in behind the reference's duck-typed solver backend (wadi2d/solver/backend.py:58-75, whose
 * members are exercised by wadi2d/solver/cpu/backend.py:14-141 and wadi2d/solver/gpu/backend.py:53-203). Each entry
 * point below names the reference member it replaces. Plain C types only: every array argument is a pointer plus a
 * size; device pointers may come from any allocator (PyTorch tensors in the package's own host layer).
 *
 * Status codes (every call returns one):
 *   W2B_OK 0, W2B_EINVAL -1 (bad argument), W2B_ECUDA -2 (a CUDA call failed), W2B_ENONFINITE -3 (a non-finite
 *   wave speed: the reference's NumericalFailure, wadi2d/solver/stepper.py:116-118), W2B_EDTMIN -4 (the step fell
 *   below dt_min, wadi2d/solver/stepper.py:119-123), W2B_ETIMEOUT -5 (a bounded device wait gave up).
 *
 * Layouts. REF_TILE is the reference's tile-with-halo state layout (wadi2d/solver/layout.py:19-50): ntiles * 1296
 * floats, tile t, row j, column i (2-cell halo). NATIVE is this library's dense layout: the padded grid with GY guard
 * rows and GX guard columns of zeros, pitch PX floats, cell (j, i) at (j + GY) * PX + i + GX; guards stand in for
 * the reference's void tile. Static per-cell and per-face arrays keep the reference's (ntiles, 32, 32) tile layout;
 * tables are repacked level-major (see w2b_pack_tables).
 *
 * Threading: one handle per stream; calls on one handle are not reentrant. The handle owns no device memory (only
 * host memory, a capture stream, three events and the device loop's graphs, all released by w2b_destroy); every
 * device buffer is the caller's and must outlive the handle. A call that fails returns no handle.
 */
#ifndef WADI_B200_H
#define WADI_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define W2B_OK 0
#define W2B_EINVAL (-1)
#define W2B_ECUDA (-2)
#define W2B_ENONFINITE (-3)
#define W2B_EDTMIN (-4)
#define W2B_ETIMEOUT (-5)

#define W2B_LAYOUT_REF_TILE 0
#define W2B_LAYOUT_NATIVE 1

/* Field ids: the state and work arrays of wadi2d/solver/layout.py:26-30 (r is not kept: it lives in shared memory). */
enum W2BField {
    W2B_H = 0, W2B_D, W2B_U, W2B_V, W2B_MX, W2B_MY, W2B_QX, W2B_QY,
    W2B_U1, W2B_V1, W2B_MX1, W2B_MY1, W2B_QX1, W2B_QY1, W2B_SRC, W2B_RES, W2B_OM, W2B_ZCX, W2B_ZCY,
    W2B_NFIELDS
};

/* Grid of wadi2d/grid/tiles.py:19-64: ny, nx padded to multiples of 32; ntiles includes the void tile 0. nruns > 1:
 * a batch of independent runs packed into one grid, each run's padded grid on its own tiles (W2BBuffers.tile_run);
 * a single run is nruns = 1. */
typedef struct {
    int32_t ny, nx, ntiles, rows, nruns;
} W2BGridDesc;

/* The native layout of a grid, from w2b_layout. */
typedef struct {
    int32_t gy, gx, px;
    int64_t ncells; /* floats per native state array: (ny + 2 gy) * px */
} W2BLayout;

/* Kernel constants: wadi2d/solver/backend.py:15-39 (NumericsRecord), plus two switches with no counterpart in the
 * reference:
 *  - level_fp64: the near-dry level of a cell (first table interval) inverted in FP64 instead of FP32 (off
 *    reproduces the reference's arithmetic);
 *  - arith: the build of the face and update passes. W2B_ARITH_EXACT is the reference's float32 arithmetic (IEEE
 *    division and square root, no FMA contraction, the correctly rounded cube root): the reference CPU twin's bits.
 *    W2B_ARITH_FAST is the same step with FMA contraction and the hardware's approximate division, square root and
 *    cube root in the face pass: fewer instructions, results within a few float32 ulp a step of the exact build's.
 *    Other values are refused with W2B_EINVAL. Changing it through w2b_set_params restarts the launch tuner. */
#define W2B_ARITH_EXACT 0
#define W2B_ARITH_FAST 1
typedef struct {
    float g, dx, e_wet, h_cfl, u_max, lead, a_min;
    int32_t second, sheet, mirror, carry, level_fp64;
    int32_t arith;
} W2BParams;

/* Device buffers (caller-owned). Ping-pong pairs [2]: the library tracks which half is current. */
typedef struct {
    /* state, NATIVE layout, ncells floats each */
    float *h[2], *u[2], *v[2], *mx[2], *my[2];
    float *d, *qx, *qy, *qx1, *qy1, *res, *src, *om, *zcx, *zcy;
    /* static, (ntiles, 32, 32) floats, reference tile layout */
    const float *hc;
    const float *fl[2], *fr[2], *gl[2], *gr[2], *ef[2], *cw[2]; /* [0] x faces, [1] y faces */
    /* tables, level-major (w2b_pack_tables): dtab2 (ntiles, rows-1, 32, 32) float2; ftab4[a] same, float4 */
    const float *dtab2;
    const float *ftab4[2];
    /* tiles: (ntiles, 2) int32 tile coordinates (tj, ti); entry 0 unused */
    const int32_t *tiles;
    /* (ny/32, nx/32) compact tile id of each tile position, 0 where none (wadi2d/grid/tiles.py:27-42) */
    const int32_t *tile_of;
    /* (ntiles, 8) neighbour tiles in the order of wadi2d/grid/tiles.py:15 */
    const int32_t *nbr;
    /* per-tile arrays (ntiles) */
    int32_t *active; /* active tile list, ntiles entries */
    float *wave;
    int32_t *wet;
    int32_t *keep;    /* tiles kept active whatever the water: sources and boundaries */
    int32_t *idle;    /* checks in a row a tile was not wanted */
    int32_t *is_act;  /* 1 on active tiles */
    int32_t *woken;   /* tiles that joined the list at the last rebuild */
    int32_t *work;    /* the device loop's work list: active tiles of the runs still stepping */
    int32_t *scratch; /* 2 * ntiles */
    /* (ntiles, 32) bit per cell: boundary cells, whose envelope entry follows the boundary overwrite */
    uint32_t *bmark;
    /* envelope, (ntiles, 32, 32) each: depth, mean depth, speed, hazard, arrival */
    float *env[5];
    /* control block, W2B_CTL_BYTES bytes, 256-byte aligned */
    void *ctl;
    /* the run table (w2b_run_table_bytes(nruns) bytes, 256-byte aligned) and the run of each tile (ntiles int32) */
    void *runs;
    const int32_t *tile_run;
    /* staging for REF_TILE transfers: ntiles * 1296 floats */
    float *stage;
    /* (ntiles) int32, or NULL: the tile of the static arrays (hc, the face scalars) and of the packed tables that each
     * tile reads. NULL: every tile its own (the arrays have ntiles tiles). Runs of a batch on one catchment can share
     * one copy: the arrays then hold only the distinct tiles (tile 0 the void tile), and table_tile maps each tile of
     * the batch to its catchment tile. No counterpart in the reference, which copies the tables into every run. */
    const int32_t *table_tile;
    /* The update pass's level cache, (ntiles, 32, 32) cells each, in tile order (not table_tile's): every cell's last
     * pair of level-table values (lpair, 2 floats a cell, 16-byte aligned) and its row (lrow, one byte a cell, 0xff:
     * none). w2b_create sets every row to 0xff. A cell whose new row is the cached one takes the cached pair, copied
     * into shared memory with the tile (coalesced), and the others gather from the table and cache what they read,
     * so the results are the table's, bit for bit. From one step to the next about one cell in 700 changes row. Valid
     * for the packed tables the handle was created with. No counterpart in the reference, which gathers every step. */
    float *lpair;
    uint8_t *lrow;
} W2BBuffers;

#define W2B_CTL_BYTES 1024

/* Stepper settings of wadi2d/solver/stepper.py:101-129 and the envelope cadence of wadi2d/engine/monitor.py:272-283. */
typedef struct {
    double cfl, wave_floor, dt_max, dt_min;
    int32_t dt_every, active_every, adaptive; /* adaptive: sleeping tiles on */
    int32_t max_every;                         /* envelope every this many steps, 0 = never */
    float arrive, deep;                        /* envelope arrival and speed depths */
} W2BStepper;

/* The stepper's state, in and out of w2b_advance: the fields of wadi2d/solver/stepper.py:24-47. */
typedef struct {
    double t, dt;
    int64_t nsteps;
    int32_t refresh_due;
    int32_t status;
    float wave_max;
    int32_t nact;
} W2BClock;

int32_t w2b_version(void);

/* Bytes of the run table of a batch of nruns runs. */
int64_t w2b_run_table_bytes(int32_t nruns);

/* Self-check of the step's float cube root (no counterpart in the reference): compares it, over count positive
 * floats from the bit pattern first_bits on, with the cube root rounded through double, as the reference's float32
 * cbrt is formed. out (device, 5 uint64, zeroed by the caller): [0] mismatches, [1..4] some mismatching inputs. */
int32_t w2b_selftest_cbrt(uint32_t first_bits, uint32_t count, uint64_t* out, void* stream);

/* Self-check of the bounded device wait (no counterpart in the reference): a barrier that nothing completes, waited on
 * for polls polls (1 <= polls <= 262144, the limit every wait of the library uses) by the library's own wait. out
 * (device, 2 int64): [0] the status the wait reports, W2B_ETIMEOUT when it gives up, as it must; [1] the SM clock
 * cycles it took. The context stays usable afterwards. */
int32_t w2b_selftest_wait(uint32_t polls, int64_t* out, void* stream);

/* Native layout of a grid. */
int32_t w2b_layout(const W2BGridDesc* grid, W2BLayout* out);

/* Native index of reference state indices (host arrays; halo entries map to the neighbour cell they copy). */
int32_t w2b_ref_to_native(const W2BGridDesc* grid, const int32_t* tiles_host, int64_t n, const int64_t* ref_index,
                          int64_t* native_index);

/* Replaces GpuBackend.__init__ (wadi2d/solver/gpu/backend.py:58-104): binds the buffers; allocates nothing on the
 * device. The caller has zeroed the state buffers and filled the static ones. */
int32_t w2b_create(const W2BGridDesc* grid, const W2BParams* params, const W2BBuffers* buffers, void** handle);
int32_t w2b_destroy(void* handle);

/* Replace the kernel constants (a new cell size or switch); the next device loop recaptures its graphs. */
int32_t w2b_set_params(void* handle, const W2BParams* params);

/* Repack reference tables (device, (ntiles,32,32,rows) and (ntiles,32,32,rows,2)) into the level-major pairs. */
int32_t w2b_pack_tables(const W2BGridDesc* grid, const float* dtab, const float* ftabx, const float* ftaby,
                        float* dtab2, float* ftab4x, float* ftab4y, void* stream);

/* Replaces set_active (wadi2d/solver/gpu/backend.py:116-119): tiles is a device array of n tile ids. */
int32_t w2b_set_active(void* handle, const int32_t* tiles, int32_t n, void* stream);

/* Replaces set_boundary (wadi2d/solver/gpu/backend.py:127-132). Device arrays of n entries; cell and ref are NATIVE
 * indices (w2b_ref_to_native). kind 0 fixed (h0, d0), 1 free, 2 follows ref lowered by d0. */
int32_t w2b_set_boundary(void* handle, int32_t n, const int32_t* cell, const int32_t* ref, const int32_t* kind,
                         const float* d0, const float* h0);

/* The boundary tally of wadi2d/engine/maxima.py:149-192: n faces (NATIVE index, axis 0 x / 1 y, sign), one FP64
 * total per face in total[n]. Device arrays. */
int32_t w2b_set_tally(void* handle, int32_t n, const int32_t* face, const int32_t* axis, const float* sign,
                      double* total);

/* Design lines (wadi2d/forcing.py:411-425 for the faces, wadi2d/engine/monitor.py:229-232 for the discharge), taken
 * every step of the device loop: line l's faces are face[start[l] .. start[l + 1]) (NATIVE index, axis 0 x / 1 y,
 * sign: +1 or -1, positive to the line's right), all in one run; q[l] = the discharge after the step (m3/s, FP64),
 * peak[l] = the largest |q[l]| so far and time[l] the time it was reached. Device arrays, kept by the caller;
 * zero peak[] to start a new search. */
int32_t w2b_set_lines(void* handle, int32_t nlines, const int32_t* start, const int32_t* face, const int32_t* axis,
                      const float* sign, double* q, double* peak, double* time);

/* Replaces step (wadi2d/solver/gpu/backend.py:151-188): faces, positivity, update, boundary, then the swap. */
int32_t w2b_step(void* handle, float dt, int32_t want_wave, int32_t want_wet, void* stream);

/* w2b_step with CUDA events around its kernels on the stream: ms[0] face pass, ms[1] update pass, ms[2] boundary
 * pass, in milliseconds (synchronises the stream). For measurement. */
int32_t w2b_step_timed(void* handle, float dt, int32_t want_wave, int32_t want_wet, void* stream, float* ms);

/* Replaces max_wave / wet_flags (wadi2d/solver/gpu/backend.py:196-200): copy to host, synchronising the stream. */
int32_t w2b_max_wave(void* handle, float* out, void* stream);
int32_t w2b_wet_flags(void* handle, int32_t* out, void* stream);

/* Replaces refresh_plan (wadi2d/solver/gpu/backend.py:139-143): tiles is a device array. */
int32_t w2b_refresh_plan(void* handle, const int32_t* tiles, int32_t n, void* stream);

/* Current device pointer of a field (ping-pong pairs resolve to their current half). The face momenta (MX, MY) are
 * not kept in their arrays while the library steps: a step's momentum is abar * u, with abar from the mean depths the
 * step started from, so the next step forms it from the other half of the mean depth pair and the face velocity
 * instead of reading it (12 bytes a cell less HBM traffic a step, the same bits). Before reading or writing U, V, MX,
 * MY (or their other halves) through this pointer, call w2b_sync_momentum on the stream that will access them; the
 * next step then starts from the arrays, written or not. MX1 and MY1 (the other halves) hold nothing between steps. */
int32_t w2b_field_ptr(void* handle, int32_t field, float** out);

/* The face momenta into their arrays (the current half of every run) and a record that the next step starts from
 * them (no work if they are there already). No counterpart in the reference, which stores the momenta every step.
 * In a batch, a momentum written for a run that does not step at the next loop step is formed from the state again
 * after it. */
int32_t w2b_sync_momentum(void* handle, void* stream);

/* Replaces get_field / set_field (wadi2d/solver/gpu/backend.py:121-125). layout REF_TILE or NATIVE; host != 0 means
 * the other pointer is host memory (pinned for an asynchronous copy). REF_TILE writes own cells only: halo entries
 * of the reference layout are copies and are read back from their owners. Both call w2b_sync_momentum first for U,
 * V, MX, MY and their other halves. */
int32_t w2b_get_field(void* handle, int32_t field, float* dst, int32_t layout, int32_t host, void* stream);
int32_t w2b_set_field(void* handle, int32_t field, const float* src, int32_t layout, int32_t host, void* stream);

/* Replaces Maxima.update (wadi2d/engine/maxima.py:118-130) over the active tiles, and Tally.add (:171-182). */
int32_t w2b_maxima(void* handle, float t, float arrive, float deep, void* stream);
int32_t w2b_tally(void* handle, double dt, void* stream);

/* Replaces the loop of Stepper.advance (wadi2d/solver/stepper.py:101-129) with a device-resident one: steps until
 * clock->t reaches t_end or max_steps steps ran, the step rule, refresh cadence, sleeping tiles, the envelope every
 * max_every steps and the boundary tally every step all on the device. clock is read and written (host memory). */
int32_t w2b_advance(void* handle, const W2BStepper* cfg, double t_end, int64_t max_steps, W2BClock* clock,
                    void* stream);

/* Rain of a source window on the device (the device form of wadi2d/forcing.py:667-683, the SCS loss of
 * wadi2d/hydrology/losses.py:69-72, and an initial-and-constant loss with no counterpart on the reference's grid
 * cells). Per rained cell m (NATIVE index cells[m]): cumulative rain P = depth[m] * f at the window's start (f0) and
 * end (f1), mm; loss 0 none, 1 SCS (s_mm, ia_mm per cell), 2 initial ia_mm then fc_mm_h; src = excess / (1000 dt).
 * partial: W2B_PARTIALS doubles of scratch. */
#define W2B_PARTIALS 296
typedef struct {
    int64_t n;
    const int32_t* cells;
    const double* depth;
    int32_t loss;
    const double* s_mm;
    const double* ia_mm;
    double fc_mm_h;
    double* partial;
} W2BRain;

/* The cell size the handle's kernels use (W2BParams.dx). */
int32_t w2b_cell_size(void* handle, float* dx);

/* Replaces Forcing.rate's rain part (wadi2d/forcing.py:667-683) for a window [t0, t1]: writes src at the rained cells
 * and volume[0] (device) = the window's rain volume, m3 (float32 rates times the cell area of each cell's run, summed
 * in FP64, times t1 - t0). */
int32_t w2b_rain_window(void* handle, const W2BRain* rain, double f0, double f1, double t0, double t1,
                        double* volume, void* stream);

/* Lumped inflows of a source window on the device: the inflow part of Forcing.rate (wadi2d/forcing.py:684-694), each
 * hydrograph's mean flow over the window shared over its cells by their level d (Injection.share,
 * wadi2d/forcing.py:468-476), which is read in place instead of copied to the host (wadi2d/forcing.py:631-644). For
 * each of n injections (n <= W2B_INFLOWS_MAX) with q[i] > 0 (q: host array, m3/s): the cells with d >= min_depth[i]
 * share q[i] in proportion to d, all of it goes to the lowest cell while none does; each cell's rate
 * (float)(q share / area) is added to src, on top of the window's rain rate where rained[cell] (the rain pass of the
 * same window wrote src there), else on 0. volume[i] (device) = injection i's window volume (its float32 rates summed
 * in FP64, times area and t1 - t0), and volume[n] += the window's total: the host form's numbers, in its order.
 *   start, lowest, min_depth: host arrays (n + 1, n, n): injection i's cells are cells[start[i] .. start[i + 1]), at
 *     most W2B_INFLOW_CELLS_MAX of them, start[0] = 0, lowest[i] the position of its lowest cell among them;
 *   cells (NATIVE indices), rained (one byte a cell): device arrays of start[n] entries; area: the cell area, m2. */
#define W2B_INFLOWS_MAX 64
#define W2B_INFLOW_CELLS_MAX 4096
typedef struct {
    int32_t n;
    const int32_t* start;
    const int32_t* lowest;
    const double* min_depth;
    const int32_t* cells;
    const uint8_t* rained;
    double area;
    double* volume;
} W2BInflow;
int32_t w2b_inflow_window(void* handle, const W2BInflow* inflow, const double* q, double t0, double t1, void* stream);

/* Uniform sources of a batch: src at each of the n NATIVE cells = rate[run of the cell] (device array of nruns,
 * m/s). The batched form of Forcing.rate's uniform rain (wadi2d/storm/uniform.py:31-35, wadi2d/forcing.py:667-683)
 * for runs that each have a storm of their own. */
int32_t w2b_source_runs(void* handle, int64_t n, const int32_t* cells, const float* rate, void* stream);

/* Replaces Monitor.storage (wadi2d/engine/monitor.py:214-218): out[0] (device) = sum of (h + res) dx^2 over the n
 * NATIVE cells, FP64, each cell read from its run's current half with its run's cell size. partial: W2B_PARTIALS
 * doubles of scratch. */
int32_t w2b_storage(void* handle, int64_t n, const int32_t* cells, double* partial, double* out, void* stream);

/* Inputs of the table builder (wadi2d/tables/builder.py:131-258; kernels of wadi2d/tables/core.py). Device pointers.
 * (ny, nx) grids are row-major float64, except mask and walls (uint8, 1 = set). Pixel (r, c) of the grid origin is
 * z[(r + row_offset) * zw + c + col_offset], indices clipped to the bed as an ArrayBed window is
 * (wadi2d/tables/builder.py:47-50). k = cell size / pixel <= 32; rows <= 64. */
typedef struct {
    const double* z;
    int64_t zh, zw;
    int32_t row_offset, col_offset;
    const double* npix; /* per-pixel Manning n aligned with z (NaN: the cell's own), or NULL */
    const double* nman; /* (ny, nx) */
    const double *xcrest, *xlen, *xc, *ycrest, *ylen, *yc; /* CrestFaces, wadi2d/tables/builder.py:62-80 */
    const uint8_t *xwall, *ywall;                         /* or NULL */
    const uint8_t* mask;
    const int32_t* tiles; /* (ntiles, 2) */
    int32_t ntiles, ny, nx, k, rows, local, margin;
    double pixel, face_depth_min, face_depth_max, beta, crest_tolerance;
} W2BTableIn;

/* Outputs: (ntiles, 32, 32[, rows[, 2]]) float32 in the reference's GridTables layout (tile 0 left as the caller
 * set it: zeros, and ones for efx, efy), and (ny, nx) float64 grids zmin, rel (mean bed over zmin), zfx, zfy (face
 * inverts) that the caller zeroed. ws: scratch of w2b_table_workspace_doubles(k + 2 margin, ws_threads) doubles,
 * ws_threads a multiple of 128 (the face kernel's thread count); needed when local != 0. */
typedef struct {
    float *hc, *dtab, *efx, *efy, *ftabx, *ftaby, *zcx, *zcy;
    float *flx, *frx, *glx, *grx, *cwx, *fly, *fry, *gly, *gry, *cwy;
    double *zmin, *rel, *zfx, *zfy;
    double* ws;
    int64_t ws_threads;
} W2BTableOut;

/* The largest W2BTableIn.margin (pixels each side of a face) the builder takes with local != 0; a negative margin or
 * a larger one is refused with W2B_EINVAL. */
#define W2B_TABLE_MARGIN_MAX (1 << 20)

/* Doubles of table-builder scratch for lines of up to nmax pixels and the given face-kernel thread count. */
int64_t w2b_table_workspace_doubles(int32_t nmax, int64_t threads);

/* Replaces build_tables (wadi2d/tables/builder.py:131-258): cell tables, face tables (strips, or the local
 * hydraulic radius when local != 0), centre beds, inverts, closed faces and natural crests, on the GPU. The local
 * radius works in shared memory when a face's line (k + 2 margin pixels) is at most about 2,800 pixels, and in
 * out->ws beyond that; out->ws is required with local != 0 either way. */
int32_t w2b_build_tables(const W2BTableIn* in, const W2BTableOut* out, void* stream);

/* w2b_build_tables for callers that cannot allocate device memory. It has no counterpart in the reference. A
 * library embedded in a host program whose device memory belongs to someone else (a pool or caching allocator it
 * does not control, a memory cap, an FFI binding with no allocator of its own) still passes its inputs and outputs,
 * but has no way to hand over the builder's scratch; this entry point allocates nothing (no cudaMalloc, cudaFree or
 * allocating library call) and uses instead a 32 MiB array of file-scope device memory, which every GPU that loads
 * the library holds until the process exits. out->ws and out->ws_threads are ignored.
 *  - Limit: a face's line (k + 2 margin pixels) of at most 3,639 pixels; longer lines are refused with W2B_EINVAL
 *    and a message. Lines that fit the builder's shared-memory workspace (up to 2,843 pixels) do not touch the array.
 *    Lines of 2,844 to 3,639 pixels do, and the array holds the workspaces of only 128 to 155 threads: the face
 *    tables are then built by a single CTA of 128 threads, correct but far slower than with a caller's workspace.
 *  - The first call on a device looks the array's address up (cudaGetSymbolAddress) with that device current;
 *    make that first call before any stream capture. The address is kept for the life of the process: it is not
 *    valid across a cudaDeviceReset.
 *  - Every call shares the one array and it keeps the last call's contents; the kernels write every scratch slot
 *    before reading it, so nothing has to start at zero. Calls that overlap on the GPU (two streams, two threads)
 *    race on it: serialise them. */
int32_t w2b_build_tables_noalloc(const W2BTableIn* in, const W2BTableOut* out, void* stream);

/* The device loop's launch schedule and its tuner. No counterpart in the reference, whose step launches each kernel
 * with one fixed grid; the tile shape stays the reference's 32 x 32 (its table layout), so what is tuned is the
 * schedule: the face pass's form, CTAs a SM of the face pass and of the update pass, and loop steps a captured graph.
 * Every configuration gives the same results bit for bit. By default the handle tunes online during its first
 * w2b_advance / w2b_advance_runs calls: successive graph launches rotate through seven candidates (the default,
 * one face-pass CTA a SM fewer, half the update pass's CTAs a SM, 8 and 32 steps a graph, and the face pass's two
 * strip forms), each timed with CUDA events from the end of the launch before it (the host's clock read between graphs
 * included) per loop step that ran; after three launches each the fastest is kept for the handle's life, the default
 * unless another is more than 2 % faster. The strip forms of the face pass take strips of 16 rows of a tile (CTAs of
 * 256 threads and 51 KB, four a SM) or of 8 rows (128 threads and 27 KB, eight a SM): the same faces bit for bit.
 * w2b_loop_tuning(h, 1, ...) starts tuning again; w2b_loop_tuning(h, tune, f, u, s) with tune 0, 2 or 3 fixes a
 * configuration with the tile form, the 16-row or the 8-row strips (1 <= f <= the form's resident CTAs a SM, 1 <= u <=
 * the update pass's, 1 <= s <= 64), W2B_EINVAL outside that. w2b_loop_config(h, out) fills out[9]: faces CTAs a SM,
 * update CTAs a SM, steps a graph (while tuning: the next launch's), tuning (1/0), the tile form's and the update
 * pass's resident CTAs a SM, the form (0 tiles, else the strip rows), and the 16-row and 8-row strip forms' resident
 * CTAs a SM. Host-driven steps (w2b_step) take the form and face-pass CTAs the tuner settled on, the tile form while
 * it tunes. */
int32_t w2b_loop_tuning(void* handle, int32_t tune, int32_t faces_per_sm, int32_t update_per_sm, int32_t steps);
int32_t w2b_loop_config(void* handle, int32_t* out);

/* Batches (W2BGridDesc.nruns > 1): each run's cell size (host array of nruns), before its first advance. */
int32_t w2b_set_run_dx(void* handle, const float* dx, int32_t n);

/* The step limiter's reading (wadi2d/solver/limiter.py:31-55 and :163-191: the CPU twin's face_step over one tile):
 * the wave speed and the new velocity of every own face of `tile` for a step `dt` from the current state, exactly as
 * the face pass would compute them, into out (device, 4096 floats: wave of the west faces, wave of the north faces,
 * new u, new v; each 32 x 32, row-major in the tile). Writes nothing else: the state is left as it was. */
int32_t w2b_face_waves(void* handle, int32_t tile, float dt, float* out, void* stream);

/* Each run's current half of the ping-pong pairs (h, u, v, mx, my): out[r] in {0, 1}, host array of nruns. In a
 * batch the runs' halves differ once their step counts do; w2b_field_ptr, w2b_get_field and w2b_set_field address
 * run 0's half. */
int32_t w2b_run_halves(void* handle, int32_t* out, void* stream);

/* The device loop over a batch: every unfinished run advances by one of its own steps per loop step, until each
 * reaches its t_end[r] (host array) or runs max_steps steps; clocks[r] in and out (host). Returns the first failing
 * status, with each run's own in clocks[r].status. */
int32_t w2b_advance_runs(void* handle, const W2BStepper* cfg, const double* t_end, int64_t max_steps,
                         W2BClock* clocks, void* stream);

/* ---- the surrogate's network (no counterpart in the reference: the storm-sweep surrogate of the critical-duration
 * search). BF16 operands are 16-bit bfloat16 arrays; every pointer is device memory. ---- */

/* c (m x n, FP32, row-major) = a (m x k, BF16, row-major) b^T (b: n x k, BF16, row-major) + bias (n, FP32, or NULL),
 * on the tensor cores (tcgen05.mma, FP32 accumulator in tensor memory). 16 <= n <= 256, n % 16 == 0, k % 16 == 0,
 * a and b 16-byte aligned. status (device int32) is set to W2B_ETIMEOUT if a bounded wait gave up. */
int32_t w2b_mma_gemm(const void* a, const void* b, int32_t m, int32_t n, int32_t k, const float* bias, float* c,
                     int32_t* status, void* stream);
/* out (BF16) = relu(z) (relu = 1) or z, n elements. */
int32_t w2b_bf16_act(const float* z, int64_t n, int32_t relu, void* out, void* stream);
/* dz (BF16) = g where z > 0, else 0. */
int32_t w2b_relu_back(const float* g, const float* z, int64_t n, void* dz, void* stream);
/* xt (cols x rows_pad, BF16) = x^T (x: rows x cols, BF16), columns past rows zero. */
int32_t w2b_transpose_bf16(const void* x, int32_t rows, int32_t cols, int32_t rows_pad, void* xt, void* stream);
/* dy (m_pad x n, BF16) = scale (y - t) on the first m rows, 0 on the rest; partial[64] (FP64) = the blocks' sums of
 * (y - t)^2. */
int32_t w2b_mse_grad(const float* y, const float* t, int32_t m, int32_t m_pad, int32_t n, float scale, void* dy,
                     double* partial, void* stream);
/* out[c] (FP32) = sum over the rows of x[r][c] (x BF16, rows x cols). */
int32_t w2b_colsum_bf16(const void* x, int32_t rows, int32_t cols, float* out, void* stream);
/* One Adam step on n FP32 weights w with gradient g and moments m, v (lr_t: the bias-corrected step size), and wb
 * (BF16, or NULL) = the new weights. */
int32_t w2b_adam(float* w, const float* g, float* m, float* v, int64_t n, float lr_t, float b1, float b2, float eps,
                 void* wb, void* stream);
/* w2b_adam with the step size read on the device: lr_t = lr_table[*step] (step: a device int64). A training step
 * captured once in a CUDA graph then replays with each step's own bias-corrected size. */
int32_t w2b_adam_table(float* w, const float* g, float* m, float* v, int64_t n, const float* lr_table,
                       const int64_t* step, float b1, float b2, float eps, void* wb, void* stream);

#ifdef __cplusplus
}
#endif

#endif
