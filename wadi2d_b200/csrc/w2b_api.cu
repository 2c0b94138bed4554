// extern "C" entry points of libwadi_b200 (declared in include/wadi_b200.h) and the host side of the handle.
//
// The handle binds caller-owned device buffers; the only memory it allocates is its own host record and the CUDA
// graphs of the device loop. Ping-pong pairs (h, u, v, mx, my) are resolved through the handle's parity, which
// flips after every step: the reference swaps its arrays the same way (wadi2d/solver/gpu/backend.py:185-188).
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include <cuda.h>

#include "w2b_common.cuh"
#include "w2b_tma.cuh"

namespace w2b {
// The face and update passes of w2b_step.cu, built twice: exact (the reference's float32 bits) and fast.
#define W2B_PASSES_DECL                                                             \
    cudaError_t faces_setup();                                                      \
    void launch_probe(const StepArgs& A, int t, float dt, float* out, cudaStream_t s); \
    int faces_occupancy();                                                          \
    void launch_faces(const TMaps& M, const StepArgs& A, int grid, cudaStream_t s); \
    cudaError_t update_setup();                                                     \
    int update_occupancy();                                                         \
    void launch_update(const TMaps& M, const StepArgs& A, int grid, cudaStream_t s); \
    int strips_occupancy(int rows);                                                 \
    void launch_strips(int rows, const TMaps& M, const StepArgs& A, int grid, cudaStream_t s);
namespace exact {
W2B_PASSES_DECL
}
namespace fast {
W2B_PASSES_DECL
}
#undef W2B_PASSES_DECL

struct Passes {
    cudaError_t (*faces_setup)();
    void (*launch_probe)(const StepArgs&, int, float, float*, cudaStream_t);
    int (*faces_occupancy)();
    void (*launch_faces)(const TMaps&, const StepArgs&, int, cudaStream_t);
    cudaError_t (*update_setup)();
    int (*update_occupancy)();
    void (*launch_update)(const TMaps&, const StepArgs&, int, cudaStream_t);
    int (*strips_occupancy)(int);
    void (*launch_strips)(int, const TMaps&, const StepArgs&, int, cudaStream_t);
};
static const Passes EXACT_PASSES = {exact::faces_setup,  exact::launch_probe,     exact::faces_occupancy,
                                    exact::launch_faces, exact::update_setup,     exact::update_occupancy,
                                    exact::launch_update, exact::strips_occupancy, exact::launch_strips};
static const Passes FAST_PASSES = {fast::faces_setup,  fast::launch_probe,     fast::faces_occupancy,
                                   fast::launch_faces, fast::update_setup,     fast::update_occupancy,
                                   fast::launch_update,  fast::strips_occupancy,  fast::launch_strips};
static const Passes& passes(const W2BParams& P) { return P.arith == W2B_ARITH_FAST ? FAST_PASSES : EXACT_PASSES; }

void launch_cbrt_check(uint32_t first, uint32_t count, unsigned long long* out, cudaStream_t s);
void launch_wait_check(uint32_t polls, long long* out, cudaStream_t s);
void launch_momentum(const StepArgs& A, int sms, cudaStream_t s);
__global__ void boundary_kernel(StepArgs A, int control);
__global__ void envelope_kernel(StepArgs A);
__global__ void control_kernel(StepArgs A);
__global__ void prestep_kernel(StepArgs A);
__global__ void setstep_kernel(StepArgs A, float dtf, int want_wave, int want_wet, int nact);
__global__ void endstep_kernel(StepArgs A);
__global__ void activity_kernel(StepArgs A, int only_work);
__global__ void plan_kernel(StepArgs A, const int32_t* list, int count);
__global__ void maxima_kernel(StepArgs A, float time, float arrive, float deep, int nact);
__global__ void tally_kernel(StepArgs A, double dt);
__global__ void ref_to_native_kernel(const float* ref, float* nat, const int32_t* tiles, int ntiles, int px);
__global__ void native_to_ref_kernel(const float* nat, float* ref, const int32_t* tiles, const int32_t* tile_of,
                                     int ntiles, int ny, int nx, int px);
__global__ void pack_tables_kernel(const float* dtab, const float* ftabx, const float* ftaby, float2* dtab2,
                                   float4* fx, float4* fy, int ntiles, int rows);
__global__ void bmark_kernel(StepArgs A, int clear_words);

// A launch configuration of the device loop: the face pass's form (whole tiles, or the strip form: half tiles in
// smaller CTAs), its CTAs a SM, the update pass's CTAs a SM, and loop steps a captured graph. Every configuration
// computes the same bits (a face's arithmetic does not depend on the form or the grid, and the wave maximum is an
// order-free integer max); they differ only in time.
struct LoopConfig {
    int faces_per_sm, update_per_sm, steps;
    int strips;  // the face pass's form: 0 whole tiles, else strips of this many rows (16 or 8)
};
constexpr int TUNE_CANDIDATES = 7;               // the default, one change of each knob either way, two strip forms
constexpr int FORCED = TUNE_CANDIDATES;          // the slot of a configuration the caller fixes
constexpr int TUNE_SAMPLES = 3;                  // timed graph launches a candidate before the tuner settles
constexpr int MAX_GRAPH_STEPS = 64;
constexpr double TUNE_MARGIN = 0.02;

// The device loop's captured graphs, one a configuration, and the online tuner that picks among them: while tuning,
// successive graph launches rotate through the candidates, each timed with CUDA events on the launching stream from
// the end of the graph before it (so the host's read of the clocks between graphs counts against the configuration
// whose graph follows it) and divided by the loop steps that ran (the empty steps of a graph that outlasts its runs
// count against the configuration that spent them). Once every candidate has TUNE_SAMPLES launches, the fastest per
// loop step is kept, the default unless another beats it by more than TUNE_MARGIN.
struct Loop {
    LoopConfig cand[TUNE_CANDIDATES + 1];
    int ncand = 0;
    cudaGraphExec_t exec[TUNE_CANDIDATES + 1] = {};
    unsigned version[TUNE_CANDIDATES + 1];
    double sec[TUNE_CANDIDATES] = {};
    long long steps[TUNE_CANDIDATES] = {};
    int samples[TUNE_CANDIDATES] = {};
    int next = 0, chosen = 0;
    int tuning = 1;
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};  // a launch's start; the ends of two successive launches
    Loop() {
        for (auto& v : version) v = ~0u;
    }
};

struct Handle {
    W2BGridDesc g{};
    W2BLayout L{};
    W2BParams P{};
    W2BBuffers B{};
    int cur = 0;  // run 0's current half (the device keeps it in R.parity[0])
    int nact = 0;
    int nruns = 1;
    RunTab R;
    int nb = 0;
    const int32_t *bcell = nullptr, *bref = nullptr, *bkind = nullptr;
    const float *bd0 = nullptr, *bh0 = nullptr;
    int ntally = 0;
    const int32_t *tface = nullptr, *taxis = nullptr;
    const float* tsign = nullptr;
    double* ttotal = nullptr;
    int nlines = 0;
    const int32_t *lstart = nullptr, *lface = nullptr, *laxis = nullptr;
    const float* lsign = nullptr;
    double *lq = nullptr, *lpeak = nullptr, *ltime = nullptr;
    int sms = 148;
    int step_blocks = 148;   // resident CTAs of the update pass
    int faces_blocks = 296;  // resident CTAs of the face pass
    int faces_occ = 2, update_occ = 1;  // resident CTAs a SM of the two passes
    int strips16_occ = 4, strips8_occ = 8;  // resident CTAs a SM of the face pass's strip forms
    TMaps tmaps;
    unsigned version = 0;   // bumped whenever a graph would capture stale arguments
    Loop loop;
    cudaStream_t cap = nullptr;  // private stream the loop graphs are captured on (a legacy stream cannot be)
    Ctl* ctl() const { return reinterpret_cast<Ctl*>(B.ctl); }
};

static StepArgs make_args(const Handle& H) {
    StepArgs A;
    memset(&A, 0, sizeof(A));
    A.P = H.P;
    A.rows = H.g.rows;
    A.px = H.L.px;
    A.ntiles = H.g.ntiles;
    A.nty = H.g.ny / TILE;
    A.ntx = H.g.nx / TILE;
    for (int q = 0; q < 2; ++q) {
        A.hh[q] = H.B.h[q];
        A.uu[0][q] = H.B.u[q];
        A.uu[1][q] = H.B.v[q];
        A.mm[0][q] = H.B.mx[q];
        A.mm[1][q] = H.B.my[q];
    }
    A.d = H.B.d;
    A.q[0] = H.B.qx;
    A.q[1] = H.B.qy;
    A.q1[0] = H.B.qx1;
    A.q1[1] = H.B.qy1;
    A.res = H.B.res;
    A.src = H.B.src;
    A.om = H.B.om;
    A.zc[0] = H.B.zcx;
    A.zc[1] = H.B.zcy;
    A.hc = H.B.hc;
    for (int a = 0; a < 2; ++a) {
        A.fl[a] = H.B.fl[a];
        A.fr[a] = H.B.fr[a];
        A.gl[a] = H.B.gl[a];
        A.gr[a] = H.B.gr[a];
        A.ef[a] = H.B.ef[a];
        A.cw[a] = H.B.cw[a];
        A.ftab4[a] = reinterpret_cast<const float4*>(H.B.ftab4[a]);
    }
    A.dtab2 = reinterpret_cast<const float2*>(H.B.dtab2);
    A.table_tile = H.B.table_tile;
    A.tiles = H.B.tiles;
    A.tile_of = H.B.tile_of;
    A.nbr = H.B.nbr;
    A.active = H.B.active;
    A.wave = H.B.wave;
    A.wet = H.B.wet;
    A.keep = H.B.keep;
    A.idle = H.B.idle;
    A.is_act = H.B.is_act;
    A.woken = H.B.woken;
    A.work = H.B.work;
    A.list = H.B.active;  // the host-driven step takes the active list; the device loop its work list
    A.scratch = H.B.scratch;
    for (int e = 0; e < 5; ++e) A.env[e] = H.B.env[e];
    A.bmark = H.B.bmark;
    A.nb = H.nb;
    A.bcell = H.bcell;
    A.bref = H.bref;
    A.bkind = H.bkind;
    A.bd0 = H.bd0;
    A.bh0 = H.bh0;
    A.ntally = H.ntally;
    A.tface = H.tface;
    A.taxis = H.taxis;
    A.tsign = H.tsign;
    A.ttotal = H.ttotal;
    A.nlines = H.nlines;
    A.lstart = H.lstart;
    A.lface = H.lface;
    A.laxis = H.laxis;
    A.lsign = H.lsign;
    A.lq = H.lq;
    A.lpeak = H.lpeak;
    A.ltime = H.ltime;
    A.ctl = H.ctl();
    A.tile_run = H.B.tile_run;
    A.lpair = reinterpret_cast<float2*>(H.B.lpair);
    A.lrow = H.B.lrow;
    A.R = H.R;
    A.nruns = H.nruns;
    return A;
}

bool handle_args(void* handle, StepArgs* out) {
    if (!handle || !out) return false;
    *out = make_args(*static_cast<Handle*>(handle));
    return true;
}

static int cuda_status(cudaError_t e, const char* where) {
    if (e == cudaSuccess) return W2B_OK;
    fprintf(stderr, "libwadi_b200: %s: %s\n", where, cudaGetErrorString(e));
    return W2B_ECUDA;
}

#define CK(call)                                              \
    do {                                                      \
        int s_ = cuda_status((call), #call);                  \
        if (s_ != W2B_OK) return s_;                          \
    } while (0)
#define CKL(where) CK(cudaGetLastError())

static int blocks_for(const Handle& H, int n) { return n < H.step_blocks ? (n > 0 ? n : 1) : H.step_blocks; }
static int faces_grid(const Handle& H, int n) { return n < H.faces_blocks ? (n > 0 ? n : 1) : H.faces_blocks; }

// cuTensorMapEncodeTiled, fetched from the driver at run time (so the library does not link libcuda).
typedef CUresult (*EncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static int encode_2d(EncodeTiled enc, CUtensorMap* map, const float* base, const W2BGridDesc& g, const W2BLayout& L,
                     uint32_t bw, uint32_t bh) {
    if (!base || ((uintptr_t)base & 15)) return W2B_EINVAL;
    const cuuint64_t dims[2] = {(cuuint64_t)L.px, (cuuint64_t)(g.ny + 2 * L.gy)};
    const cuuint64_t strides[1] = {(cuuint64_t)L.px * 4};
    const cuuint32_t box[2] = {bw, bh};
    const cuuint32_t es[2] = {1, 1};
    const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void*)base, dims, strides, box, es,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        fprintf(stderr, "libwadi_b200: cuTensorMapEncodeTiled failed (%d)\n", (int)r);
        return W2B_ECUDA;
    }
    return W2B_OK;
}

static int build_tmaps(Handle& H) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn ||
        q != cudaDriverEntryPointSuccess)
        return W2B_ECUDA;
    EncodeTiled enc = reinterpret_cast<EncodeTiled>(fn);
    const W2BBuffers& B = H.B;
    int st = W2B_OK;
    auto box = [&](CUtensorMap* m, const float* p) {
        if (st == W2B_OK) st = encode_2d(enc, m, p, H.g, H.L, 40, 36);
    };
    auto own = [&](CUtensorMap* m, const float* p) {
        if (st == W2B_OK) st = encode_2d(enc, m, p, H.g, H.L, 32, 32);
    };
    box(&H.tmaps.d, B.d);
    box(&H.tmaps.qx, B.qx);
    box(&H.tmaps.qy, B.qy);
    box(&H.tmaps.om, B.om);
    box(&H.tmaps.zcx, B.zcx);
    box(&H.tmaps.zcy, B.zcy);
    box(&H.tmaps.qx1, B.qx1);
    box(&H.tmaps.qy1, B.qy1);
    own(&H.tmaps.res, B.res);
    own(&H.tmaps.src, B.src);
    for (int p = 0; p < 2; ++p) {
        box(&H.tmaps.h[p], B.h[p]);
        box(&H.tmaps.u[p], B.u[p]);
        box(&H.tmaps.v[p], B.v[p]);
        own(&H.tmaps.mx[p], B.mx[p]);
        own(&H.tmaps.my[p], B.my[p]);
    }
    // the strip forms' boxes, 40 columns of the rows the face arithmetic reads around a strip of `rows` rows: the
    // velocities rows + 4 (two above, two below), the y discharge rows + 2, the x lip rows, depth, mean depth, x
    // discharge and y lip rows + 1 (one above); 32 x rows for the momenta
    for (const int rows : {16, 8}) {
        StripMaps& S = rows == 16 ? H.tmaps.s16 : H.tmaps.s8;
        auto strip = [&](CUtensorMap* m, const float* q, int extra) {
            if (st == W2B_OK) st = encode_2d(enc, m, q, H.g, H.L, 40, (uint32_t)(rows + extra));
        };
        auto strip_own = [&](CUtensorMap* m, const float* q) {
            if (st == W2B_OK) st = encode_2d(enc, m, q, H.g, H.L, 32, (uint32_t)rows);
        };
        strip(&S.d, B.d, 1);
        strip(&S.qx, B.qx, 1);
        strip(&S.qy, B.qy, 2);
        strip(&S.zcx, B.zcx, 0);
        strip(&S.zcy, B.zcy, 1);
        for (int p = 0; p < 2; ++p) {
            strip(&S.h[p], B.h[p], 1);
            strip(&S.u[p], B.u[p], 4);
            strip(&S.v[p], B.v[p], 4);
            strip_own(&S.mx[p], B.mx[p]);
            strip_own(&S.my[p], B.my[p]);
        }
    }
    return st;
}

static void drop_graph(Handle& H, int c) {
    if (H.loop.exec[c]) {
        cudaGraphExecDestroy(H.loop.exec[c]);
        H.loop.exec[c] = nullptr;
    }
    H.loop.version[c] = ~0u;
}

static void drop_graphs(Handle& H) {
    for (int c = 0; c <= TUNE_CANDIDATES; ++c) drop_graph(H, c);
}

// The tuner's candidates: the occupancy-given default (both passes at their resident CTAs a SM, 16 steps a graph),
// and from it one CTA a SM fewer in the face pass, half the update pass's, 8 and 32 steps a graph, and the face pass
// in its strip form at its resident CTAs a SM.
static void init_loop(Handle& H) {
    Loop& L = H.loop;
    const int F = H.faces_occ, U = H.update_occ;
    L.ncand = 0;
    L.cand[L.ncand++] = {F, U, 16, 0};
    if (F > 1) L.cand[L.ncand++] = {F - 1, U, 16, 0};
    if (U > 1) L.cand[L.ncand++] = {F, (U + 1) / 2, 16, 0};
    L.cand[L.ncand++] = {F, U, 8, 0};
    L.cand[L.ncand++] = {F, U, 32, 0};
    L.cand[L.ncand++] = {H.strips16_occ, U, 16, 16};
    L.cand[L.ncand++] = {H.strips8_occ, U, 16, 8};
    L.cand[FORCED] = L.cand[0];
    for (int c = 0; c < TUNE_CANDIDATES; ++c) {
        L.sec[c] = 0.0;
        L.steps[c] = 0;
        L.samples[c] = 0;
    }
    L.next = L.chosen = 0;
    L.tuning = 1;
}

// CTAs of boundary_kernel: enough for its items (boundary cells; with control, tally faces and a warp a line), at
// most four a SM.
static int boundary_grid(const Handle& H, int control) {
    int64_t items = H.nb;
    if (control) {
        items = items > H.ntally ? items : H.ntally;
        items = items > (int64_t)H.nlines * 32 ? items : (int64_t)H.nlines * 32;
    }
    int64_t g = (items + 255) / 256;
    const int64_t cap = 4 * (int64_t)(H.sms > 0 ? H.sms : 148);
    return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

// The shared-memory limits of both builds' passes, and the resident CTAs a SM of the handle's build (W2BParams.arith),
// which set the launch grids and the tuner's candidates.
static int set_passes(Handle& H) {
    for (const Passes* X : {&EXACT_PASSES, &FAST_PASSES}) {
        if (X->update_setup() != cudaSuccess || X->faces_setup() != cudaSuccess)
            return cuda_status(cudaGetLastError(), "pass setup");
    }
    const Passes& X = passes(H.P);
    const int occ = X.update_occupancy(), focc = X.faces_occupancy();
    const int s16 = X.strips_occupancy(16), s8 = X.strips_occupancy(8);
    H.update_occ = occ > 0 ? occ : 1;
    H.faces_occ = focc > 0 ? focc : 1;
    H.strips16_occ = s16 > 0 ? s16 : 1;
    H.strips8_occ = s8 > 0 ? s8 : 1;
    H.step_blocks = H.sms * H.update_occ;
    H.faces_blocks = H.sms * H.faces_occ;
    init_loop(H);
    return W2B_OK;
}

// The face pass of a host-driven step (w2b_step, w2b_step_timed) over n tiles: in the form and at the CTAs a SM the
// device loop's tuner settled on, the tile form while it tunes.
static void launch_faces_host(Handle& H, const StepArgs& A, int n, cudaStream_t s) {
    const LoopConfig& C = H.loop.cand[H.loop.chosen];
    if (!H.loop.tuning && C.strips) {
        const int g = H.sms * C.faces_per_sm, units = (TILE / C.strips) * n;
        passes(H.P).launch_strips(C.strips, H.tmaps, A, units < g ? units : g, s);
    } else {
        passes(H.P).launch_faces(H.tmaps, A, faces_grid(H, n), s);
    }
}

// One step of the device loop under launch configuration C: every running run advances by one of its own steps.
static int launch_loop_step(Handle& H, const LoopConfig& C, cudaStream_t s) {
    StepArgs A = make_args(H);
    A.list = A.work;
    const dim3 blk(32, 8);
    const int grid = blocks_for(H, H.g.ntiles - 1);
    const int tiles = H.g.ntiles - 1 > 0 ? H.g.ntiles - 1 : 1;
    const int fgrid = H.sms * C.faces_per_sm, ugrid = H.sms * C.update_per_sm;
    const Passes& X = passes(H.P);
    if (C.strips)
        X.launch_strips(C.strips, H.tmaps, A, (TILE / C.strips) * tiles < fgrid ? (TILE / C.strips) * tiles : fgrid, s);
    else
        X.launch_faces(H.tmaps, A, tiles < fgrid ? tiles : fgrid, s);
    X.launch_update(H.tmaps, A, tiles < ugrid ? tiles : ugrid, s);
    envelope_kernel<<<H.sms * 2, TILE2, 0, s>>>(A);
    boundary_kernel<<<boundary_grid(H, 1), 256, 0, s>>>(A, 1);
    control_kernel<<<1, 1024, 0, s>>>(A);  // clocks, rebuild and work list, the next step's settings
    plan_kernel<<<grid, blk, 0, s>>>(A, A.woken, -1);
    CKL("loop step");
    return W2B_OK;
}

}  // namespace w2b

using namespace w2b;

extern "C" {

int32_t w2b_version(void) { return 3; }

int64_t w2b_run_table_bytes(int32_t nruns) { return nruns < 1 ? 0 : (int64_t)run_table_bytes(nruns); }

int32_t w2b_selftest_cbrt(uint32_t first_bits, uint32_t count, uint64_t* out, void* stream) {
    if (!out) return W2B_EINVAL;
    launch_cbrt_check(first_bits, count, reinterpret_cast<unsigned long long*>(out), (cudaStream_t)stream);
    CKL("w2b_selftest_cbrt");
    return W2B_OK;
}

int32_t w2b_selftest_wait(uint32_t polls, int64_t* out, void* stream) {
    if (!out || polls < 1 || polls > TMA_WAIT_LIMIT) return W2B_EINVAL;
    launch_wait_check(polls, reinterpret_cast<long long*>(out), (cudaStream_t)stream);
    CKL("w2b_selftest_wait");
    return W2B_OK;
}

int32_t w2b_layout(const W2BGridDesc* grid, W2BLayout* out) {
    if (!grid || !out || grid->ny <= 0 || grid->nx <= 0 || grid->ny % TILE || grid->nx % TILE || grid->ntiles < 1)
        return W2B_EINVAL;
    out->gy = GY;
    out->gx = GX;
    out->px = grid->nx + 2 * GX;
    out->ncells = (int64_t)(grid->ny + 2 * GY) * out->px;
    return W2B_OK;
}

int32_t w2b_ref_to_native(const W2BGridDesc* grid, const int32_t* tiles_host, int64_t n, const int64_t* ref_index,
                          int64_t* native_index) {
    W2BLayout L;
    if (w2b_layout(grid, &L) != W2B_OK || !tiles_host || n < 0 || (n && (!ref_index || !native_index)))
        return W2B_EINVAL;
    for (int64_t m = 0; m < n; ++m) {
        const int64_t k = ref_index[m];
        const int64_t t = k / 1296;
        if (k < 0 || t < 1 || t >= grid->ntiles) return W2B_EINVAL;
        const int64_t r = k % 1296;
        const int64_t j = (int64_t)tiles_host[2 * t] * TILE + r / 36 - 2;
        const int64_t i = (int64_t)tiles_host[2 * t + 1] * TILE + r % 36 - 2;
        native_index[m] = (j + L.gy) * L.px + i + L.gx;
    }
    return W2B_OK;
}

int32_t w2b_create(const W2BGridDesc* grid, const W2BParams* params, const W2BBuffers* buffers, void** handle) {
    if (!grid || !params || !buffers || !handle) return W2B_EINVAL;
    if (grid->rows < 4 || grid->rows > 64 || grid->nruns < 1) return W2B_EINVAL;
    if (params->arith != W2B_ARITH_EXACT && params->arith != W2B_ARITH_FAST) return W2B_EINVAL;
    if (!buffers->runs || ((uintptr_t)buffers->runs & 255) || !buffers->tile_run || !buffers->work) return W2B_EINVAL;
    {
        // arrays the passes stage with bulk copies: 16-byte aligned
        auto a16 = [](const void* q) { return q && !((uintptr_t)q & 15); };
        bool ok = a16(buffers->hc) && a16(buffers->lpair) && a16(buffers->lrow);
        for (int x = 0; x < 2; ++x)
            ok = ok && a16(buffers->fl[x]) && a16(buffers->fr[x]) && a16(buffers->gl[x]) && a16(buffers->gr[x]) &&
                 a16(buffers->ef[x]) && a16(buffers->cw[x]);
        for (int e = 0; e < 5; ++e) ok = ok && a16(buffers->env[e]);
        if (!ok) return W2B_EINVAL;
    }
    Handle* H = new (std::nothrow) Handle();
    if (!H) return W2B_EINVAL;
    H->g = *grid;
    H->P = *params;
    H->B = *buffers;
    if (w2b_layout(grid, &H->L) != W2B_OK || !H->B.ctl || ((uintptr_t)H->B.ctl & 255)) {
        delete H;
        return W2B_EINVAL;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&H->sms, cudaDevAttrMultiProcessorCount, dev);
    if (set_passes(*H) != W2B_OK) {
        delete H;
        return W2B_ECUDA;
    }
    if (build_tmaps(*H) != W2B_OK) {
        delete H;
        return W2B_ECUDA;
    }
    H->nact = grid->ntiles - 1;
    H->nruns = grid->nruns;
    H->R = run_table(H->B.runs, H->nruns);
    // the level cache holds nothing yet: every row 0xff
    if (cudaMemset(H->B.lrow, 0xff, (size_t)H->g.ntiles * TILE2) != cudaSuccess) {
        delete H;
        return cuda_status(cudaGetLastError(), "w2b_create level cache");
    }
    const int32_t stored = 1;  // the caller's momentum arrays hold the momenta the first step starts from
    if (cudaMemcpy(&H->ctl()->m_stored, &stored, sizeof(stored), cudaMemcpyHostToDevice) != cudaSuccess) {
        delete H;
        return cuda_status(cudaGetLastError(), "w2b_create control block");
    }
    if (H->nruns == 1 && cudaMemcpy(H->R.dx, &H->P.dx, sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
        delete H;
        return cuda_status(cudaGetLastError(), "w2b_create run table");
    }
    if (cudaStreamCreateWithFlags(&H->cap, cudaStreamNonBlocking) != cudaSuccess) {
        delete H;
        return cuda_status(cudaGetLastError(), "w2b_create stream");
    }
    if (cudaEventCreate(&H->loop.ev[0]) != cudaSuccess || cudaEventCreate(&H->loop.ev[1]) != cudaSuccess ||
        cudaEventCreate(&H->loop.ev[2]) != cudaSuccess) {
        for (auto& e : H->loop.ev)
            if (e) cudaEventDestroy(e);
        cudaStreamDestroy(H->cap);
        delete H;
        return cuda_status(cudaGetLastError(), "w2b_create events");
    }
    const int st = cuda_status(cudaGetLastError(), "w2b_create");
    if (st != W2B_OK) {  // no handle goes out with a failure: the caller has nothing to destroy
        w2b_destroy(H);
        return st;
    }
    *handle = H;
    return W2B_OK;
}

int32_t w2b_destroy(void* handle) {
    if (!handle) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    drop_graphs(*H);
    for (auto& e : H->loop.ev)
        if (e) cudaEventDestroy(e);
    if (H->cap) cudaStreamDestroy(H->cap);
    delete H;
    return W2B_OK;
}

int32_t w2b_pack_tables(const W2BGridDesc* grid, const float* dtab, const float* ftabx, const float* ftaby,
                        float* dtab2, float* ftab4x, float* ftab4y, void* stream) {
    if (!grid || !dtab || !ftabx || !ftaby || !dtab2 || !ftab4x || !ftab4y || grid->rows < 4) return W2B_EINVAL;
    if (((uintptr_t)dtab2 & 7) || ((uintptr_t)ftab4x & 15) || ((uintptr_t)ftab4y & 15)) return W2B_EINVAL;
    pack_tables_kernel<<<1024, 256, 0, (cudaStream_t)stream>>>(dtab, ftabx, ftaby, reinterpret_cast<float2*>(dtab2),
                                                              reinterpret_cast<float4*>(ftab4x),
                                                              reinterpret_cast<float4*>(ftab4y), grid->ntiles,
                                                              grid->rows);
    CKL("w2b_pack_tables");
    return W2B_OK;
}

int32_t w2b_set_params(void* handle, const W2BParams* params) {
    if (!handle || !params) return W2B_EINVAL;
    if (params->arith != W2B_ARITH_EXACT && params->arith != W2B_ARITH_FAST) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    const int arith = H->P.arith;
    H->P = *params;
    H->version++;
    if (params->arith != arith) {  // the other build's passes: their occupancy, and the tuner starts again
        drop_graphs(*H);
        const int st = set_passes(*H);
        if (st != W2B_OK) return st;
    }
    if (H->nruns == 1) CK(cudaMemcpy(H->R.dx, &H->P.dx, sizeof(float), cudaMemcpyHostToDevice));
    return W2B_OK;
}

int32_t w2b_set_active(void* handle, const int32_t* tiles, int32_t n, void* stream) {
    if (!handle || n < 0) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    if (n > H->g.ntiles - 1 || (n && !tiles)) return W2B_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    if (n && tiles != H->B.active)
        CK(cudaMemcpyAsync(H->B.active, tiles, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s));
    H->nact = n;
    return W2B_OK;
}

int32_t w2b_set_boundary(void* handle, int32_t n, const int32_t* cell, const int32_t* ref, const int32_t* kind,
                         const float* d0, const float* h0) {
    if (!handle || n < 0 || (n && (!cell || !ref || !kind || !d0 || !h0))) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    H->nb = n;
    H->bcell = cell;
    H->bref = ref;
    H->bkind = kind;
    H->bd0 = d0;
    H->bh0 = h0;
    H->version++;
    const StepArgs A = make_args(*H);
    bmark_kernel<<<64, 256>>>(A, H->g.ntiles * TILE);
    if (n) bmark_kernel<<<64, 256>>>(A, 0);
    CKL("w2b_set_boundary");
    return W2B_OK;
}

int32_t w2b_set_tally(void* handle, int32_t n, const int32_t* face, const int32_t* axis, const float* sign,
                      double* total) {
    if (!handle || n < 0 || (n && (!face || !axis || !sign || !total))) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    H->ntally = n;
    H->tface = face;
    H->taxis = axis;
    H->tsign = sign;
    H->ttotal = total;
    H->version++;
    return W2B_OK;
}

int32_t w2b_set_lines(void* handle, int32_t nlines, const int32_t* start, const int32_t* face, const int32_t* axis,
                      const float* sign, double* q, double* peak, double* time) {
    if (!handle || nlines < 0 || (nlines && (!start || !face || !axis || !sign || !q || !peak || !time)))
        return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    H->nlines = nlines;
    H->lstart = start;
    H->lface = face;
    H->laxis = axis;
    H->lsign = sign;
    H->lq = q;
    H->lpeak = peak;
    H->ltime = time;
    H->version++;
    return W2B_OK;
}

int32_t w2b_step(void* handle, float dt, int32_t want_wave, int32_t want_wet, void* stream) {
    if (!handle) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    cudaStream_t s = (cudaStream_t)stream;
    if (H->nruns != 1) return W2B_EINVAL;  // a batch steps in the device loop
    if (want_wave) CK(cudaMemsetAsync(H->B.wave, 0, sizeof(float) * H->g.ntiles, s));
    const StepArgs A = make_args(*H);
    setstep_kernel<<<1, 1, 0, s>>>(A, dt, want_wave, want_wet, H->nact);
    if (H->nact == 0) {  // as the reference: no tiles, no swap
        CKL("w2b_step");
        return W2B_OK;
    }
    const int grid = blocks_for(*H, H->nact);
    launch_faces_host(*H, A, H->nact, s);
    passes(H->P).launch_update(H->tmaps, A, grid, s);
    if (H->nb) boundary_kernel<<<boundary_grid(*H, 0), 256, 0, s>>>(A, 0);
    endstep_kernel<<<1, 1, 0, s>>>(A);
    CKL("w2b_step");
    H->cur ^= 1;
    return W2B_OK;
}

int32_t w2b_step_timed(void* handle, float dt, int32_t want_wave, int32_t want_wet, void* stream, float* ms) {
    if (!handle || !ms) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    cudaStream_t s = (cudaStream_t)stream;
    if (H->nact == 0 || H->nruns != 1) return W2B_EINVAL;
    cudaEvent_t ev[4];
    for (auto& e : ev) CK(cudaEventCreate(&e));
    if (want_wave) CK(cudaMemsetAsync(H->B.wave, 0, sizeof(float) * H->g.ntiles, s));
    const StepArgs A = make_args(*H);
    setstep_kernel<<<1, 1, 0, s>>>(A, dt, want_wave, want_wet, H->nact);
    const int grid = blocks_for(*H, H->nact);
    CK(cudaEventRecord(ev[0], s));
    launch_faces_host(*H, A, H->nact, s);
    CK(cudaEventRecord(ev[1], s));
    passes(H->P).launch_update(H->tmaps, A, grid, s);
    CK(cudaEventRecord(ev[2], s));
    if (H->nb) boundary_kernel<<<boundary_grid(*H, 0), 256, 0, s>>>(A, 0);
    endstep_kernel<<<1, 1, 0, s>>>(A);
    CK(cudaEventRecord(ev[3], s));
    CKL("w2b_step_timed");
    H->cur ^= 1;
    CK(cudaEventSynchronize(ev[3]));
    for (int e = 0; e < 3; ++e) CK(cudaEventElapsedTime(ms + e, ev[e], ev[e + 1]));
    for (auto& e : ev) cudaEventDestroy(e);
    return W2B_OK;
}

int32_t w2b_max_wave(void* handle, float* out, void* stream) {
    if (!handle || !out) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    int32_t status = 0;
    CK(cudaMemcpyAsync(out, H->R.wave_bits, sizeof(float), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    CK(cudaMemcpyAsync(&status, &H->ctl()->status, sizeof(int32_t), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    CK(cudaStreamSynchronize((cudaStream_t)stream));
    return status == W2B_ETIMEOUT ? W2B_ETIMEOUT : W2B_OK;
}

int32_t w2b_wet_flags(void* handle, int32_t* out, void* stream) {
    if (!handle || !out) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    CK(cudaMemcpyAsync(out, H->B.wet, sizeof(int32_t) * H->g.ntiles, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    CK(cudaStreamSynchronize((cudaStream_t)stream));
    return W2B_OK;
}

int32_t w2b_refresh_plan(void* handle, const int32_t* tiles, int32_t n, void* stream) {
    if (!handle || n < 0 || (n && !tiles)) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    if (!n) return W2B_OK;
    const StepArgs A = make_args(*H);
    plan_kernel<<<blocks_for(*H, n), dim3(32, 8), 0, (cudaStream_t)stream>>>(A, tiles, n);
    CKL("w2b_refresh_plan");
    return W2B_OK;
}

static float* field_ptr(Handle* H, int f) {
    const int c = H->cur, o = 1 - H->cur;
    switch (f) {
        case W2B_H: return H->B.h[c];
        case W2B_D: return H->B.d;
        case W2B_U: return H->B.u[c];
        case W2B_V: return H->B.v[c];
        case W2B_MX: return H->B.mx[c];
        case W2B_MY: return H->B.my[c];
        case W2B_QX: return H->B.qx;
        case W2B_QY: return H->B.qy;
        case W2B_U1: return H->B.u[o];
        case W2B_V1: return H->B.v[o];
        case W2B_MX1: return H->B.mx[o];
        case W2B_MY1: return H->B.my[o];
        case W2B_QX1: return H->B.qx1;
        case W2B_QY1: return H->B.qy1;
        case W2B_SRC: return H->B.src;
        case W2B_RES: return H->B.res;
        case W2B_OM: return H->B.om;
        case W2B_ZCX: return H->B.zcx;
        case W2B_ZCY: return H->B.zcy;
        default: return nullptr;
    }
}

int32_t w2b_cell_size(void* handle, float* dx) {
    if (!handle || !dx) return W2B_EINVAL;
    *dx = static_cast<Handle*>(handle)->P.dx;
    return W2B_OK;
}

int32_t w2b_field_ptr(void* handle, int32_t field, float** out) {
    if (!handle || !out) return W2B_EINVAL;
    float* p = field_ptr(static_cast<Handle*>(handle), field);
    if (!p) return W2B_EINVAL;
    *out = p;
    return W2B_OK;
}

// Fields whose reading or writing needs the momenta in their arrays: the momenta themselves, and the velocities they
// are formed from (a velocity written afterwards must not change the momentum the next step starts from).
static bool momentum_field(int f) {
    return f == W2B_U || f == W2B_V || f == W2B_MX || f == W2B_MY || f == W2B_U1 || f == W2B_V1 || f == W2B_MX1 ||
           f == W2B_MY1;
}

static int sync_momentum(Handle& H, cudaStream_t s) {
    launch_momentum(make_args(H), H.sms, s);
    CKL("w2b_sync_momentum");
    return W2B_OK;
}

int32_t w2b_get_field(void* handle, int32_t field, float* dst, int32_t layout, int32_t host, void* stream) {
    if (!handle || !dst) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    float* src = field_ptr(H, field);
    if (!src) return W2B_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    if (momentum_field(field)) {
        const int st = sync_momentum(*H, s);
        if (st != W2B_OK) return st;
    }
    if (layout == W2B_LAYOUT_NATIVE) {
        CK(cudaMemcpyAsync(dst, src, sizeof(float) * H->L.ncells,
                           host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s));
    } else if (layout == W2B_LAYOUT_REF_TILE) {
        float* out = host ? H->B.stage : dst;
        native_to_ref_kernel<<<H->g.ntiles, 256, 0, s>>>(src, out, H->B.tiles, H->B.tile_of, H->g.ntiles, H->g.ny,
                                                         H->g.nx, H->L.px);
        CKL("native_to_ref");
        if (host)
            CK(cudaMemcpyAsync(dst, out, sizeof(float) * 1296 * (size_t)H->g.ntiles, cudaMemcpyDeviceToHost, s));
    } else {
        return W2B_EINVAL;
    }
    if (host) CK(cudaStreamSynchronize(s));
    return W2B_OK;
}

int32_t w2b_set_field(void* handle, int32_t field, const float* src, int32_t layout, int32_t host, void* stream) {
    if (!handle || !src) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    float* dst = field_ptr(H, field);
    if (!dst) return W2B_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    if (momentum_field(field)) {
        const int st = sync_momentum(*H, s);
        if (st != W2B_OK) return st;
    }
    if (layout == W2B_LAYOUT_NATIVE) {
        CK(cudaMemcpyAsync(dst, src, sizeof(float) * H->L.ncells,
                           host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));
    } else if (layout == W2B_LAYOUT_REF_TILE) {
        const float* in = src;
        if (host) {
            CK(cudaMemcpyAsync(H->B.stage, src, sizeof(float) * 1296 * (size_t)H->g.ntiles, cudaMemcpyHostToDevice,
                               s));
            in = H->B.stage;
        }
        ref_to_native_kernel<<<H->g.ntiles - 1 > 0 ? H->g.ntiles - 1 : 1, 256, 0, s>>>(in, dst, H->B.tiles,
                                                                                       H->g.ntiles, H->L.px);
        CKL("ref_to_native");
    } else {
        return W2B_EINVAL;
    }
    if (host) CK(cudaStreamSynchronize(s));
    return W2B_OK;
}

int32_t w2b_sync_momentum(void* handle, void* stream) {
    if (!handle) return W2B_EINVAL;
    return sync_momentum(*static_cast<Handle*>(handle), (cudaStream_t)stream);
}

int32_t w2b_maxima(void* handle, float t, float arrive, float deep, void* stream) {
    if (!handle) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    if (!H->nact) return W2B_OK;
    const StepArgs A = make_args(*H);
    maxima_kernel<<<blocks_for(*H, H->nact), dim3(32, 8), 0, (cudaStream_t)stream>>>(A, t, arrive, deep, H->nact);
    CKL("w2b_maxima");
    return W2B_OK;
}

int32_t w2b_tally(void* handle, double dt, void* stream) {
    if (!handle) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    if (!H->ntally) return W2B_OK;
    const StepArgs A = make_args(*H);
    tally_kernel<<<(H->ntally + 255) / 256, 256, 0, (cudaStream_t)stream>>>(A, dt);
    CKL("w2b_tally");
    return W2B_OK;
}

// The graph of configuration c, captured again when the arguments it would hold have changed.
static int loop_graph(Handle& H, int c) {
    Loop& L = H.loop;
    if (L.exec[c] && L.version[c] == H.version) return W2B_OK;
    drop_graph(H, c);
    cudaGraph_t graph;
    CK(cudaStreamBeginCapture(H.cap, cudaStreamCaptureModeThreadLocal));
    int stc = W2B_OK;
    for (int k = 0; k < L.cand[c].steps && stc == W2B_OK; ++k) stc = launch_loop_step(H, L.cand[c], H.cap);
    cudaError_t e = cudaStreamEndCapture(H.cap, &graph);
    if (stc != W2B_OK) {
        if (e == cudaSuccess) cudaGraphDestroy(graph);
        return stc;
    }
    CK(e);
    e = cudaGraphInstantiate(&L.exec[c], graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) L.exec[c] = nullptr;  // nothing to destroy later
    CK(e);
    L.version[c] = H.version;
    return W2B_OK;
}

// One timed launch of candidate c ran `live` loop steps in `ms`: add it, move to the next candidate, and settle on the
// fastest once every candidate has its samples.
static void tune_sample(Handle& H, int c, long long live, float ms) {
    Loop& L = H.loop;
    if (live > 0) {
        L.sec[c] += 1e-3 * (double)ms;
        L.steps[c] += live;
        L.samples[c] += 1;
    }
    L.next = (c + 1) % L.ncand;
    for (int k = 0; k < L.ncand; ++k)
        if (L.samples[k] < TUNE_SAMPLES) return;
    auto per_step = [&](int k) { return L.sec[k] / (double)(L.steps[k] > 0 ? L.steps[k] : 1); };
    int best = 0;
    for (int k = 1; k < L.ncand; ++k)
        if (per_step(k) < per_step(best)) best = k;
    if (best != 0 && !(per_step(best) < (1.0 - TUNE_MARGIN) * per_step(0))) best = 0;
    L.chosen = best;
    L.tuning = 0;
    for (int k = 0; k < L.ncand; ++k)
        if (k != best) drop_graph(H, k);
}

// A single run's loop settings and clock, written by one thread from its arguments. A copy from the host would be
// queued on a copy engine behind any large upload in flight on another stream (the next window's source, staged while
// this window steps) and wait for it; kernel arguments travel with the launch. The stored-momenta flag stays.
__global__ void advance_setup_kernel(Ctl c, double t, double dt, double t_end, long long nsteps, long long max_steps,
                                     int32_t refresh_due, Ctl* ctl, RunTab R) {
    c.m_stored = ctl->m_stored;
    *ctl = c;
    R.t[0] = t;
    R.dt[0] = dt;
    R.t_end[0] = t_end;
    R.nsteps[0] = nsteps;
    R.steps_run[0] = 0;
    R.max_steps[0] = max_steps;
    R.refresh_due[0] = refresh_due;
    R.status[0] = 0;
}

// The device-resident loop. Steps run in chunks of a captured graph (the launch configuration's steps), every running
// run advancing one of its own steps each graph step; after each chunk the host reads the runs' clocks once.
static int advance_runs(Handle* H, const W2BStepper* cfg, const double* t_end, int64_t max_steps, W2BClock* clocks,
                        cudaStream_t s) {
    const int n = H->nruns;
    Ctl c;
    memset(&c, 0, sizeof(c));
    c.nact = H->nact;
    c.nruns = n;
    c.dt_every = cfg->dt_every;
    c.active_every = cfg->active_every;
    c.adaptive = cfg->adaptive;
    c.max_every = cfg->max_every;
    c.arrive = cfg->arrive;
    c.deep = cfg->deep;
    c.cfl = cfg->cfl;
    c.wave_floor = cfg->wave_floor;
    c.dt_max = cfg->dt_max;
    c.dt_min = cfg->dt_min;
    std::vector<double> t(n), dt(n), te(t_end, t_end + n);
    std::vector<long long> ns(n), zero(n, 0), ms(n, (long long)max_steps);
    std::vector<int32_t> rd(n), st(n, 0);
    for (int r = 0; r < n; ++r) {
        t[r] = clocks[r].t;
        dt[r] = clocks[r].dt;
        ns[r] = clocks[r].nsteps;
        rd[r] = clocks[r].refresh_due;
    }
    const RunTab& R = H->R;
    if (n == 1) {  // by kernel arguments: no host-to-device copy (see advance_setup_kernel)
        advance_setup_kernel<<<1, 1, 0, s>>>(c, t[0], dt[0], te[0], ns[0], ms[0], rd[0], H->ctl(), R);
        CKL("advance settings");
    } else {
        CK(cudaMemcpyAsync(H->ctl(), &c, offsetof(Ctl, m_stored), cudaMemcpyHostToDevice, s));  // the flag stays
        CK(cudaMemcpyAsync(R.t, t.data(), 8 * n, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(R.dt, dt.data(), 8 * n, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(R.t_end, te.data(), 8 * n, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(R.nsteps, ns.data(), 8 * n, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(R.steps_run, zero.data(), 8 * n, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(R.max_steps, ms.data(), 8 * n, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(R.refresh_due, rd.data(), 4 * n, cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(R.status, st.data(), 4 * n, cudaMemcpyHostToDevice, s));
    }
    activity_kernel<<<1, 1024, 0, s>>>(make_args(*H), 1);  // the work list of the runs that take a step
    prestep_kernel<<<1, 1024, 0, s>>>(make_args(*H));      // the first step's settings; each step sets the next's
    CKL("advance work list");
    Loop& L = H->loop;
    std::vector<long long> run(n);
    long long ran_before = 0;  // loop steps so far in this call (the largest steps_run of any run)
    int32_t gstatus = 0;
    int end = 1, have_prev = 0;  // ev[end] takes this launch's end; ev[3 - end] holds the last one's, if have_prev
    if (L.tuning)  // every candidate's graph before the first timed launch: no capture falls inside a timing
        for (int k = 0; k < L.ncand; ++k) {
            const int stc = loop_graph(*H, k);
            if (stc != W2B_OK) return stc;
        }
    for (;;) {
        const bool timed = L.tuning != 0;
        const int c = timed ? L.next : L.chosen;
        const int stc = loop_graph(*H, c);
        if (stc != W2B_OK) return stc;
        if (timed && !have_prev) CK(cudaEventRecord(L.ev[0], s));
        CK(cudaGraphLaunch(L.exec[c], s));
        if (timed) CK(cudaEventRecord(L.ev[end], s));
        CK(cudaMemcpyAsync(t.data(), R.t, 8 * n, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(run.data(), R.steps_run, 8 * n, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(st.data(), R.status, 4 * n, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(&gstatus, &H->ctl()->status, 4, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (timed) {
            long long ran = 0;
            for (int r = 0; r < n; ++r) ran = run[r] > ran ? run[r] : ran;
            float ms = 0.0f;
            CK(cudaEventElapsedTime(&ms, have_prev ? L.ev[3 - end] : L.ev[0], L.ev[end]));
            tune_sample(*H, c, ran - ran_before, ms);
            ran_before = ran;
            have_prev = 1;
            end = 3 - end;
        } else {
            have_prev = 0;
        }
        bool done = gstatus != 0;
        if (!done) {
            done = true;
            for (int r = 0; r < n; ++r)
                if (st[r] == 0 && t[r] < te[r] - 1e-9 && run[r] < ms[r]) done = false;
        }
        if (done) break;
    }
    std::vector<uint32_t> wb(n);
    std::vector<int32_t> par(n);
    CK(cudaMemcpyAsync(dt.data(), R.dt, 8 * n, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(ns.data(), R.nsteps, 8 * n, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(wb.data(), R.wave_last, 4 * n, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(par.data(), R.parity, 4 * n, cudaMemcpyDeviceToHost, s));
    int32_t nact = 0;
    CK(cudaMemcpyAsync(&nact, &H->ctl()->nact, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    H->nact = nact;
    H->cur = par[0];
    int32_t first = gstatus;
    for (int r = 0; r < n; ++r) {
        clocks[r].t = t[r];
        clocks[r].dt = dt[r];
        clocks[r].nsteps = ns[r];
        clocks[r].refresh_due = 0;
        clocks[r].status = st[r] != 0 ? st[r] : gstatus;
        float w;
        memcpy(&w, &wb[r], 4);
        clocks[r].wave_max = w;
        clocks[r].nact = nact;
        if (!first && st[r]) first = st[r];
    }
    return first;
}

int32_t w2b_advance(void* handle, const W2BStepper* cfg, double t_end, int64_t max_steps, W2BClock* clock,
                    void* stream) {
    if (!handle || !cfg || !clock || max_steps < 0 || cfg->dt_every < 1 || cfg->active_every < 1) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    if (H->nruns != 1) return W2B_EINVAL;
    return advance_runs(H, cfg, &t_end, max_steps, clock, (cudaStream_t)stream);
}

int32_t w2b_advance_runs(void* handle, const W2BStepper* cfg, const double* t_end, int64_t max_steps,
                         W2BClock* clocks, void* stream) {
    if (!handle || !cfg || !clocks || !t_end || max_steps < 0 || cfg->dt_every < 1 || cfg->active_every < 1)
        return W2B_EINVAL;
    return advance_runs(static_cast<Handle*>(handle), cfg, t_end, max_steps, clocks, (cudaStream_t)stream);
}

int32_t w2b_loop_tuning(void* handle, int32_t tune, int32_t faces_per_sm, int32_t update_per_sm, int32_t steps) {
    if (!handle) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    Loop& L = H->loop;
    if (tune == 1) {
        drop_graphs(*H);
        init_loop(*H);
        return W2B_OK;
    }
    if (tune < 0 || tune > 3) return W2B_EINVAL;
    const int strips = tune == 2 ? 16 : (tune == 3 ? 8 : 0);
    const int occ = strips == 16 ? H->strips16_occ : (strips == 8 ? H->strips8_occ : H->faces_occ);
    if (faces_per_sm < 1 || faces_per_sm > occ || update_per_sm < 1 ||
        update_per_sm > H->update_occ || steps < 1 || steps > MAX_GRAPH_STEPS)
        return W2B_EINVAL;
    L.cand[FORCED] = {faces_per_sm, update_per_sm, steps, strips};
    drop_graph(*H, FORCED);
    L.chosen = FORCED;
    L.tuning = 0;
    return W2B_OK;
}

int32_t w2b_loop_config(void* handle, int32_t* out) {
    if (!handle || !out) return W2B_EINVAL;
    const Handle* H = static_cast<const Handle*>(handle);
    const Loop& L = H->loop;
    const LoopConfig& C = L.cand[L.tuning ? L.next : L.chosen];
    out[0] = C.faces_per_sm;
    out[1] = C.update_per_sm;
    out[2] = C.steps;
    out[3] = L.tuning;
    out[4] = H->faces_occ;
    out[5] = H->update_occ;
    out[6] = C.strips;
    out[7] = H->strips16_occ;
    out[8] = H->strips8_occ;
    return W2B_OK;
}

int32_t w2b_face_waves(void* handle, int32_t tile, float dt, float* out, void* stream) {
    if (!handle || !out || !(dt > 0.0f)) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    if (tile < 1 || tile >= H->g.ntiles) return W2B_EINVAL;
    passes(H->P).launch_probe(make_args(*H), tile, dt, out, (cudaStream_t)stream);
    CKL("w2b_face_waves");
    return W2B_OK;
}

int32_t w2b_run_halves(void* handle, int32_t* out, void* stream) {
    if (!handle || !out) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    cudaStream_t s = (cudaStream_t)stream;
    CK(cudaMemcpyAsync(out, H->R.parity, sizeof(int32_t) * H->nruns, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return W2B_OK;
}

int32_t w2b_set_run_dx(void* handle, const float* dx, int32_t n) {
    if (!handle || !dx) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    if (n != H->nruns) return W2B_EINVAL;
    CK(cudaMemcpy(H->R.dx, dx, sizeof(float) * n, cudaMemcpyHostToDevice));
    return W2B_OK;
}

}  // extern "C"
