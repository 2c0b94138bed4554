// extern "C" entry points of libwadi_b200 (declared in include/wadi_b200.h) and the host side of the handle.
//
// The handle binds caller-owned device buffers; the only memory it allocates is its own host record and the CUDA
// graphs of the device loop. Ping-pong pairs (h, u, v, mx, my) are resolved through the handle's parity, which
// flips after every step: the reference swaps its arrays the same way (wadi2d/solver/gpu/backend.py:185-188).
#include <cstdio>
#include <cstring>
#include <new>

#include <cuda.h>

#include "w2b_common.cuh"

namespace w2b {
cudaError_t faces_setup();
void launch_cbrt_check(uint32_t first, uint32_t count, unsigned long long* out, cudaStream_t s);
int faces_occupancy();
void launch_faces(const TMaps& M, const StepArgs& A, int p, int grid, cudaStream_t s);
cudaError_t update_setup();
int update_occupancy();
void launch_update(const TMaps& M, const StepArgs& A, int p, int grid, cudaStream_t s);
__global__ void boundary_kernel(StepArgs A, int control);
__global__ void prestep_kernel(Ctl* ctl);
__global__ void setstep_kernel(Ctl* ctl, float dtf, int want_wave, int want_wet, int nact);
__global__ void activity_kernel(StepArgs A);
__global__ void plan_kernel(StepArgs A, const int32_t* list, int count, const float* h);
__global__ void maxima_kernel(StepArgs A, float time, float arrive, float deep, int nact);
__global__ void tally_kernel(StepArgs A, double dt);
__global__ void ref_to_native_kernel(const float* ref, float* nat, const int32_t* tiles, int ntiles, int px);
__global__ void native_to_ref_kernel(const float* nat, float* ref, const int32_t* tiles, const int32_t* tile_of,
                                     int ntiles, int ny, int nx, int px);
__global__ void pack_tables_kernel(const float* dtab, const float* ftabx, const float* ftaby, float2* dtab2,
                                   float4* fx, float4* fy, int ntiles, int rows);
__global__ void bmark_kernel(StepArgs A, int clear_words);

struct Loop {
    cudaGraphExec_t exec[2] = {nullptr, nullptr};  // by starting parity
    int steps = 0;
    unsigned version = ~0u;
};

struct Handle {
    W2BGridDesc g{};
    W2BLayout L{};
    W2BParams P{};
    W2BBuffers B{};
    int cur = 0;
    int nact = 0;
    int nb = 0;
    const int32_t *bcell = nullptr, *bref = nullptr, *bkind = nullptr;
    const float *bd0 = nullptr, *bh0 = nullptr;
    int ntally = 0;
    const int32_t *tface = nullptr, *taxis = nullptr;
    const float* tsign = nullptr;
    double* ttotal = nullptr;
    int sms = 148;
    int step_blocks = 148;   // resident CTAs of the update pass
    int faces_blocks = 296;  // resident CTAs of the face pass
    TMaps tmaps;
    unsigned version = 0;   // bumped whenever a graph would capture stale arguments
    Loop loop;
    cudaStream_t cap = nullptr;  // private stream the loop graphs are captured on (a legacy stream cannot be)
    Ctl* ctl() const { return reinterpret_cast<Ctl*>(B.ctl); }
};

static StepArgs make_args(const Handle& H, int p) {
    StepArgs A;
    memset(&A, 0, sizeof(A));
    const int n = 1 - p;
    A.P = H.P;
    A.rows = H.g.rows;
    A.px = H.L.px;
    A.ntiles = H.g.ntiles;
    A.nty = H.g.ny / TILE;
    A.ntx = H.g.nx / TILE;
    A.area = H.P.dx * H.P.dx;
    A.h = H.B.h[p];
    A.h_next = H.B.h[n];
    A.u[0] = H.B.u[p];
    A.u[1] = H.B.v[p];
    A.u_next[0] = H.B.u[n];
    A.u_next[1] = H.B.v[n];
    A.m[0] = H.B.mx[p];
    A.m[1] = H.B.my[p];
    A.m_next[0] = H.B.mx[n];
    A.m_next[1] = H.B.my[n];
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
    A.ctl = H.ctl();
    return A;
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
    return st;
}

static void drop_graphs(Handle& H) {
    for (auto& e : H.loop.exec)
        if (e) {
            cudaGraphExecDestroy(e);
            e = nullptr;
        }
    H.loop.version = ~0u;
}

// One step of the device loop, parity p.
static int launch_loop_step(Handle& H, int p, cudaStream_t s) {
    const StepArgs A = make_args(H, p);
    const dim3 blk(32, 8);
    const int grid = blocks_for(H, H.g.ntiles - 1);
    prestep_kernel<<<1, 1, 0, s>>>(A.ctl);
    launch_faces(H.tmaps, A, p, faces_grid(H, H.g.ntiles - 1), s);
    launch_update(H.tmaps, A, p, grid, s);
    boundary_kernel<<<1, 256, 0, s>>>(A, 1);
    activity_kernel<<<1, 1024, 0, s>>>(A);
    plan_kernel<<<grid, blk, 0, s>>>(A, A.woken, -1, A.h_next);
    CKL("loop step");
    return W2B_OK;
}

}  // namespace w2b

using namespace w2b;

extern "C" {

int32_t w2b_version(void) { return 1; }

int32_t w2b_selftest_cbrt(uint32_t first_bits, uint32_t count, uint64_t* out, void* stream) {
    if (!out) return W2B_EINVAL;
    launch_cbrt_check(first_bits, count, reinterpret_cast<unsigned long long*>(out), (cudaStream_t)stream);
    CKL("w2b_selftest_cbrt");
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
    if (grid->rows < 4 || grid->rows > 64) return W2B_EINVAL;
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
    if (update_setup() != cudaSuccess) {
        delete H;
        return cuda_status(cudaGetLastError(), "w2b_create update_setup");
    }
    const int occ = update_occupancy();
    H->step_blocks = H->sms * (occ > 0 ? occ : 1);
    if (faces_setup() != cudaSuccess) {
        delete H;
        return cuda_status(cudaGetLastError(), "w2b_create faces_setup");
    }
    const int focc = faces_occupancy();
    H->faces_blocks = H->sms * (focc > 0 ? focc : 1);
    if (build_tmaps(*H) != W2B_OK) {
        delete H;
        return W2B_ECUDA;
    }
    H->nact = grid->ntiles - 1;
    if (cudaStreamCreateWithFlags(&H->cap, cudaStreamNonBlocking) != cudaSuccess) {
        delete H;
        return cuda_status(cudaGetLastError(), "w2b_create stream");
    }
    *handle = H;
    return cuda_status(cudaGetLastError(), "w2b_create");
}

int32_t w2b_destroy(void* handle) {
    if (!handle) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    drop_graphs(*H);
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
    Handle* H = static_cast<Handle*>(handle);
    H->P = *params;
    H->version++;
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
    const StepArgs A = make_args(*H, H->cur);
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

int32_t w2b_step(void* handle, float dt, int32_t want_wave, int32_t want_wet, void* stream) {
    if (!handle) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    cudaStream_t s = (cudaStream_t)stream;
    if (want_wave) CK(cudaMemsetAsync(H->B.wave, 0, sizeof(float) * H->g.ntiles, s));
    setstep_kernel<<<1, 1, 0, s>>>(H->ctl(), dt, want_wave, want_wet, H->nact);
    if (H->nact == 0) {
        CKL("w2b_step");
        return W2B_OK;
    }
    const StepArgs A = make_args(*H, H->cur);
    const int grid = blocks_for(*H, H->nact);
    launch_faces(H->tmaps, A, H->cur, faces_grid(*H, H->nact), s);
    launch_update(H->tmaps, A, H->cur, grid, s);
    if (H->nb) boundary_kernel<<<1, 256, 0, s>>>(A, 0);
    CKL("w2b_step");
    H->cur ^= 1;
    return W2B_OK;
}

int32_t w2b_step_timed(void* handle, float dt, int32_t want_wave, int32_t want_wet, void* stream, float* ms) {
    if (!handle || !ms) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    cudaStream_t s = (cudaStream_t)stream;
    if (H->nact == 0) return W2B_EINVAL;
    cudaEvent_t ev[4];
    for (auto& e : ev) CK(cudaEventCreate(&e));
    if (want_wave) CK(cudaMemsetAsync(H->B.wave, 0, sizeof(float) * H->g.ntiles, s));
    setstep_kernel<<<1, 1, 0, s>>>(H->ctl(), dt, want_wave, want_wet, H->nact);
    const StepArgs A = make_args(*H, H->cur);
    const int grid = blocks_for(*H, H->nact);
    CK(cudaEventRecord(ev[0], s));
    launch_faces(H->tmaps, A, H->cur, faces_grid(*H, H->nact), s);
    CK(cudaEventRecord(ev[1], s));
    launch_update(H->tmaps, A, H->cur, grid, s);
    CK(cudaEventRecord(ev[2], s));
    if (H->nb) boundary_kernel<<<1, 256, 0, s>>>(A, 0);
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
    CK(cudaMemcpyAsync(out, &H->ctl()->wave_max, sizeof(float), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
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
    const StepArgs A = make_args(*H, H->cur);
    plan_kernel<<<blocks_for(*H, n), dim3(32, 8), 0, (cudaStream_t)stream>>>(A, tiles, n, H->B.h[H->cur]);
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

int32_t w2b_get_field(void* handle, int32_t field, float* dst, int32_t layout, int32_t host, void* stream) {
    if (!handle || !dst) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    float* src = field_ptr(H, field);
    if (!src) return W2B_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
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

int32_t w2b_maxima(void* handle, float t, float arrive, float deep, void* stream) {
    if (!handle) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    if (!H->nact) return W2B_OK;
    StepArgs A = make_args(*H, H->cur);
    A.u_next[0] = H->B.u[H->cur];  // the envelope reads the state after the step
    A.u_next[1] = H->B.v[H->cur];
    maxima_kernel<<<blocks_for(*H, H->nact), dim3(32, 8), 0, (cudaStream_t)stream>>>(A, t, arrive, deep, H->nact);
    CKL("w2b_maxima");
    return W2B_OK;
}

int32_t w2b_tally(void* handle, double dt, void* stream) {
    if (!handle) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    if (!H->ntally) return W2B_OK;
    const StepArgs A = make_args(*H, H->cur);
    tally_kernel<<<(H->ntally + 255) / 256, 256, 0, (cudaStream_t)stream>>>(A, dt);
    CKL("w2b_tally");
    return W2B_OK;
}

// The device-resident loop. Steps run in chunks of a captured graph of LOOP_STEPS steps (an even number, so a chunk
// that runs to its end leaves the parity where it found it); after each chunk the host reads the clock once.
static constexpr int LOOP_STEPS = 16;

int32_t w2b_advance(void* handle, const W2BStepper* cfg, double t_end, int64_t max_steps, W2BClock* clock,
                    void* stream) {
    if (!handle || !cfg || !clock || max_steps < 0 || cfg->dt_every < 1 || cfg->active_every < 1) return W2B_EINVAL;
    Handle* H = static_cast<Handle*>(handle);
    cudaStream_t s = (cudaStream_t)stream;
    // clock and settings into the control block
    Ctl init;
    CK(cudaMemcpyAsync(&init, H->ctl(), sizeof(Ctl), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    init.t = clock->t;
    init.dt = clock->dt;
    init.t_end = t_end;
    init.nsteps = clock->nsteps;
    init.steps_run = 0;
    init.max_steps = max_steps;
    init.refresh_due = clock->refresh_due;
    init.status = 0;
    init.nact = H->nact;
    init.ticket = 0u;
    init.run = 1;
    init.cfl = cfg->cfl;
    init.wave_floor = cfg->wave_floor;
    init.dt_max = cfg->dt_max;
    init.dt_min = cfg->dt_min;
    init.dx = (double)H->P.dx;
    init.dt_every = cfg->dt_every;
    init.active_every = cfg->active_every;
    init.adaptive = cfg->adaptive;
    init.max_every = cfg->max_every;
    init.arrive = cfg->arrive;
    init.deep = cfg->deep;
    init.want_max = 0;
    CK(cudaMemcpyAsync(H->ctl(), &init, sizeof(Ctl), cudaMemcpyHostToDevice, s));
    // graphs for both starting parities, rebuilt when an argument they captured has changed
    if (H->loop.version != H->version) {
        drop_graphs(*H);
        for (int p0 = 0; p0 < 2; ++p0) {
            cudaGraph_t graph;
            CK(cudaStreamBeginCapture(H->cap, cudaStreamCaptureModeThreadLocal));
            int st = W2B_OK;
            for (int k = 0; k < LOOP_STEPS && st == W2B_OK; ++k) st = launch_loop_step(*H, (p0 + k) & 1, H->cap);
            cudaError_t e = cudaStreamEndCapture(H->cap, &graph);
            if (st != W2B_OK) return st;
            CK(e);
            e = cudaGraphInstantiate(&H->loop.exec[p0], graph, 0);
            cudaGraphDestroy(graph);
            CK(e);
        }
        H->loop.version = H->version;
    }
    Ctl now;
    long long done = 0;
    for (;;) {
        CK(cudaGraphLaunch(H->loop.exec[H->cur], s));
        CK(cudaMemcpyAsync(&now, H->ctl(), sizeof(Ctl), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        const long long ran = now.steps_run - done;
        done = now.steps_run;
        H->cur ^= (int)(ran & 1);
        if (now.status != 0 || !(now.t < t_end - 1e-9) || now.steps_run >= max_steps || ran < LOOP_STEPS) break;
    }
    H->nact = now.nact;
    clock->t = now.t;
    clock->dt = now.dt;
    clock->nsteps = now.nsteps;
    clock->refresh_due = 0;
    clock->status = now.status;
    clock->wave_max = now.wave_max;
    clock->nact = now.nact;
    return now.status;
}

}  // extern "C"
