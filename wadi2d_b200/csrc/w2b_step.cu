// The uniform-grid step on sm_100a: face pass, update pass (positivity ratio, continuity, level lookup), envelope pass,
// boundary/tally/control pass, active-list rebuild, and the layout converters.
//
// A CTA takes one 32 x 32 tile at a time, looping over its share of the work list (grid-stride, so a graph-captured
// launch serves any list length): the face pass with 512 threads (a thread a column, two rows), the update pass with
// 256 (a thread a column, four rows). State sits in the dense NATIVE layout, so a neighbour is an address offset and
// the reference's halo exchanges (wadi2d/solver/gpu/kernels/cells.cu:80-93) disappear; the guard ring is zero like
// the reference's void tile. In a batch every tile reads its run's clock, cell size, flags and current half.
//
// The face pass restates wadi2d/solver/gpu/kernels/faces.cu:10-175 (= wadi2d/solver/cpu/kernels.py:86-244); the
// update pass fuses limit and update (cells.cu:4-63, kernels.py:247-299) by computing the positivity ratio r of the
// tile and its one-cell ring in shared memory; the boundary pass restates cells.cu:95-111 and engine/maxima.py:53-62.
#include <cstdio>

#include "w2b_common.cuh"
#include "w2b_tma.cuh"

namespace w2b {

// The face and update passes are compiled twice (wadi2d_b200/build.py): into namespace exact with the library's IEEE
// flags, the reference's float32 bits, and into namespace fast with W2B_FAST and FMA contraction (the approximate
// division, square root and cube root and the hardware max and min of w2b_common.cuh qdiv/qsqrt/qcbrt/qmax/qmin, in
// the face arithmetic). W2BParams.arith picks one per handle.
// Everything after them (envelope, boundary, control, converters) is compiled once, with the exact build.
#ifdef W2B_FAST
#define W2B_ARITH fast
#else
#define W2B_ARITH exact
#endif
namespace W2B_ARITH {

// ------------------------------------------------------------------ face pass

// Shared-memory image of one tile for the face pass. Boxes of 40 x 36 floats hold the tile with 2 cells of halo north
// and south and 4 west and east (the TMA box starts on a 16-byte boundary); own cell (j, i) sits at box (j + 2, i + 4).
constexpr int BOXW = 40, BOXH = 36, BOX = BOXW * BOXH;
constexpr int F_D = 0, F_H = 1, F_U = 2, F_V = 3, F_QX = 4, F_QY = 5, F_OM = 6, F_ZCX = 7, F_ZCY = 8, NBOX = 9;
constexpr int SM_M = NBOX * BOX;          // mx, my: 32 x 32 each
constexpr int SM_ST = SM_M + 2 * TILE2;   // the 12 static face scalars of the tile, 32 x 32 each
constexpr int SM_FLOATS = SM_ST + 12 * TILE2;
constexpr int FACES_SMEM = SM_FLOATS * 4;  // 109,184 bytes: two CTAs a SM
constexpr int FACES_THREADS = 512;

// The two images the face helpers read. off(f) is the offset of state field f's array as the helpers index it, by
// box index b (b's row 0 is two rows above the tile's or strip's first row, its column 0 four columns west of the
// first column; a row is BOXW floats). A whole tile (the face pass and the probe): nine 40 x 36 boxes, the plan share
// among them. A strip (the strip forms of the face pass): each state field's box holds only the rows the face
// arithmetic reads, the plan share is read from global memory on the refresh steps that want it. S is the stride of a
// static face scalar's (and of a momentum's) array in the image: 1,024 floats for a tile, 32 H for a strip.
struct TileImage {
    static constexpr int M = SM_M, ST = SM_ST, S = TILE2;
    static constexpr int HO = SM_M;  // the last step's mean depth box (40 x 36), in the momenta's place
    static constexpr bool OM = true;
    __host__ __device__ static constexpr int off(int f) { return f * BOX; }
};
__host__ __device__ constexpr int pad32(int n) { return (n + 31) / 32 * 32; }  // floats, to a 128-byte boundary
template <int H>
struct StripImage {
    // The rows of each field's box around a strip of H rows, from the face arithmetic's reads (b - S, b, b + S,
    // b +- 2 S, b +- PP, b +- 2 PP of face_in, face_a, face_bc): the velocities two rows above to two below; depth,
    // mean depth, x discharge and the y lip one row above to the last row; the y discharge one above to one below;
    // the x lip the strip's own rows.
    static constexpr int R_UV = H + 4, R_QY = H + 2, R_ZCX = H, R_1 = H + 1;
    // each box's region, 128-byte aligned, in the order u v d h qx qy zcx zcy (u first: every offset is >= 0)
    static constexpr int S_U = 0, S_V = S_U + pad32(BOXW * R_UV), S_D = S_V + pad32(BOXW * R_UV);
    static constexpr int S_H = S_D + pad32(BOXW * R_1), S_QX = S_H + pad32(BOXW * R_1);
    static constexpr int S_QY = S_QX + pad32(BOXW * R_1), S_ZCX = S_QY + pad32(BOXW * R_QY);
    static constexpr int S_ZCY = S_ZCX + pad32(BOXW * R_ZCX), S_END = S_ZCY + pad32(BOXW * R_1);
    static constexpr int M = S_END, ST = S_END + 2 * TILE * H, S = TILE * H;
    // the last step's mean depth box, in the momenta's place: the rows of the mean depth's box, BOXW * (H + 1) <=
    // 2 TILE H floats
    static constexpr int HO = M - BOXW;
    static constexpr bool OM = false;
    static constexpr int FLOATS = ST + 12 * S;
    static constexpr int SMEM = FLOATS * 4;        // 51,840 bytes for 16 rows (four CTAs a SM), 27,264 for 8 (eight)
    // the bytes the strip's copies bring (the regions without their padding): with the momenta, or with the last
    // step's mean depth in their place
    static constexpr int BYTES = 4 * (BOXW * (2 * R_UV + 4 * R_1 + R_QY + R_ZCX) + 14 * TILE * H);
    static constexpr int BYTES_HO = BYTES - 4 * (2 * TILE * H - BOXW * R_1);
    static constexpr int THREADS = 16 * H;         // a warp two rows
    static constexpr int CTAS = H == 16 ? 4 : 8;   // resident CTAs a SM the launch bound plans for
    __host__ __device__ static constexpr int off(int f) {
        return f == F_U   ? S_U
             : f == F_V   ? S_V
             : f == F_D   ? S_D - BOXW
             : f == F_H   ? S_H - BOXW
             : f == F_QX  ? S_QX - BOXW
             : f == F_QY  ? S_QY - BOXW
             : f == F_ZCX ? S_ZCX - 2 * BOXW
                          : S_ZCY - BOXW;
    }
};
static_assert(StripImage<8>::SMEM == 27264 && StripImage<16>::SMEM == 51840, "strip image sizes");
static_assert(StripImage<8>::off(F_D) >= 0 && StripImage<8>::off(F_ZCX) >= 0, "strip offsets");
static_assert(BOXW * StripImage<8>::R_1 <= 2 * TILE * 8 && BOXW * StripImage<16>::R_1 <= 2 * TILE * 16 &&
                  BOX <= 2 * TILE2,
              "the last step's mean depth box fits the momenta's place");

// What the first part of a face hands to the rest: the row's quad (its load is issued in part A and consumed after
// the table-free momentum terms), the face depth, and the table row with the upwind choice, the live flag and the
// above-the-table flag packed in one word. Parts B and C re-read the other inputs from the tile's image, so few
// registers stay live across the momentum terms.
struct FaceA {
    float4 q;
    float eface;
    int bits;
};
constexpr int FA_ROW = 0xff, FA_LEFT = 0x100, FA_LIVE = 0x200, FA_ABOVE = 0x400;

// The face's upwind inputs from the tile's image (wadi2d/solver/gpu/kernels/faces.cu:19-31): the levels over each
// side's invert, their positive parts, and the velocity on the face.
struct FaceIn {
    float e_l, e_r, e_lp, e_rp, uf;
};
template <int AX, class L>
__device__ __forceinline__ FaceIn face_in(const float* sm, int b, int sl) {
    constexpr int S = AX == 0 ? 1 : BOXW;
    const float* D = sm + L::off(F_D);
    const float* U = sm + L::off(AX == 0 ? F_U : F_V);
    const float* st = sm + L::ST + AX * 6 * L::S;
    FaceIn I;
    I.e_l = D[b - S] - st[0 * L::S + sl];
    I.e_r = D[b] - st[1 * L::S + sl];
    I.uf = U[b];
    I.e_lp = qmax(I.e_l, 0.0f);
    I.e_rp = qmax(I.e_r, 0.0f);
    return I;
}

// Part A of the face of axis AX at box index b (wadi2d/solver/gpu/kernels/faces.cu:19-44).
// ON: the numerics switches (second-order momentum, sheet flow, dry-face mirroring, depth carry) are all on, as the
// reference's defaults have them, and known to the compiler; otherwise they are read from A.P.
// L: the image (TileImage, StripImage); sl: the cell's index in the image's static arrays, local: in the tile.
template <int AX, bool ON = false, class L = TileImage>
__device__ __forceinline__ void face_a(const float* sm, int b, int sl, int local, const StepArgs& A, int t,
                                       FaceA& F) {
    constexpr int S = AX == 0 ? 1 : BOXW;
    const W2BParams& P = A.P;
    const float* st = sm + L::ST + AX * 6 * L::S;
    const FaceIn I = face_in<AX, L>(sm, b, sl);
    const bool from_left = I.uf > 0.0f || (I.uf == 0.0f && I.e_l >= I.e_r);
    const float eup = from_left ? I.e_lp : I.e_rp;
    F.bits = from_left ? FA_LEFT : 0;
    if (eup <= P.e_wet) return;
    const float cwf = st[5 * L::S + sl];
    const float top = st[4 * L::S + sl];
    float eface = eup;
    if ((ON || P.carry) && cwf == 0.0f) {
        const float* ZC = sm + L::off(AX == 0 ? F_ZCX : F_ZCY);
        const float dz = from_left ? ZC[b - S] - st[0 * L::S + sl] : ZC[b] - st[1 * L::S + sl];
        if (dz > 1e-6f) {
            float phi = qdiv(eup - 2.0f * dz, 2.0f * dz);
            phi = phi < 0.0f ? 0.0f : (phi > 1.0f ? 1.0f : phi);
            eface = eup - phi * dz;
        }
    }
    const int last = A.rows - 1;
    const bool above = eface >= top;
    const int r = above ? last - 1 : row_of(qsqrt(qdiv(eface, top)) * (float)last, last);
    F.eface = eface;
    F.bits |= FA_LIVE | (above ? FA_ABOVE : 0) | r;
    const float4* quads = A.ftab4[AX] + (size_t)t * (A.rows - 1) * TILE2 + local;
    F.q = __ldg(quads + (size_t)r * TILE2);
}

// Parts B and C: the momentum terms (faces.cu:50-100, table-free), then the lookup, section, friction, crest cap,
// outputs and wave speed (faces.cu:43-44, :52-63, :102-145). Returns the wave speed.
// mst: the face's momentum is the image's stored one (Ctl::m_stored), else it is formed from the last step's mean
// depths (the image's HO box) and the face velocity, as the step that wrote the velocity formed it. The new momentum
// is not written: the next step forms it the same way.
// PROBE: write the face's new velocity to probe_un[local] and nothing of the state (the step-limiter probe).
template <int AX, bool PROBE = false, bool ON = false, class L = TileImage>
__device__ __forceinline__ float face_bc(const float* sm, int b, int sl, int local, int k, const StepArgs& A, int t,
                                         const FaceA& F, float dt, float dx, int want_wave, const float* rowc, int p,
                                         int mst, float* probe_un = nullptr) {
    constexpr int S = AX == 0 ? 1 : BOXW;
    constexpr int PP = AX == 0 ? BOXW : 1;
    const W2BParams& P = A.P;
    if (!(F.bits & FA_LIVE)) {
        if constexpr (PROBE) {
            probe_un[local] = 0.0f;
        } else {
            A.uu[AX][1 - p][k] = 0.0f;
            A.q1[AX][k] = 0.0f;
        }
        return 0.0f;
    }
    const float ZERO = 0.0f, HALF = 0.5f, ONE = 1.0f;
    const float span = dx;
    const float* H = sm + L::off(F_H);
    const float* U = sm + L::off(AX == 0 ? F_U : F_V);
    const float* VP = sm + L::off(AX == 0 ? F_V : F_U);
    const float* Q = sm + L::off(AX == 0 ? F_QX : F_QY);
    const float* QP = sm + L::off(AX == 0 ? F_QY : F_QX);
    const float* st = sm + L::ST + AX * 6 * L::S;
    const FaceIn I = face_in<AX, L>(sm, b, sl);
    const bool from_left = (F.bits & FA_LEFT) != 0;
    const float uf = I.uf;
    const float eup = from_left ? I.e_lp : I.e_rp;
    const float h_l = H[b - S], h_r = H[b];
    const float hup = from_left ? h_l : h_r;

    // [1] section: the disconnected drive (the volume-limited section needs the table, below)
    float d_eta = I.e_rp - I.e_lp;
    if (ON || P.sheet) {
        const float edown = from_left ? I.e_rp : I.e_lp;
        if (edown <= ZERO) {
            const float g_u = from_left ? st[2 * L::S + sl] : st[3 * L::S + sl];
            const float g_d = from_left ? st[3 * L::S + sl] : st[2 * L::S + sl];
            const float h_d = from_left ? h_r : h_l;
            const float drop = (hup - g_u) - qmax(h_d - g_d, HALF * (g_u - g_d));
            const float level_drop = fabsf(I.e_l - I.e_r);
            const float drive = qmax(eup, qmin(drop, level_drop));
            d_eta = from_left ? -drive : drive;
        }
    }
    // [3] momentum fluxes
    const int mirror = ON ? 1 : P.mirror, second = ON ? 1 : P.second;
    const float um = gated(U[b - S], uf, mirror);
    const float up = gated(U[b + S], uf, mirror);
    const float umm = gated(U[b - 2 * S], um, mirror);
    const float upp = gated(U[b + 2 * S], up, mirror);
    const float qk = Q[b];
    const float qc_l = HALF * (Q[b - S] + qk);
    const float qc_r = HALF * (qk + Q[b + S]);
    // each upwind choice picks the arguments of one ustar (the same value as choosing between two ustar calls)
    const bool pl = qc_l > ZERO, pr = qc_r > ZERO;
    const float s_l = ustar(pl ? um : uf, pl ? umm : up, pl ? uf : um, second);
    const float s_r = ustar(pr ? uf : up, pr ? um : upp, pr ? up : uf, second);
    float flux = qc_r * s_r - qc_l * s_l;
    const float qy_s = HALF * (QP[b - S] + QP[b]);
    const float qy_n = HALF * (QP[b - S + PP] + QP[b + PP]);
    const float u_s = gated(U[b - PP], uf, mirror);
    const float u_n = gated(U[b + PP], uf, mirror);
    const float uss = gated(U[b - 2 * PP], u_s, mirror);
    const float unn = gated(U[b + 2 * PP], u_n, mirror);
    const bool ps = qy_s > ZERO, pn = qy_n > ZERO;
    const float us_s = ustar(ps ? u_s : uf, ps ? uss : u_n, ps ? uf : u_s, second);
    const float us_n = ustar(pn ? uf : u_n, pn ? u_s : unn, pn ? u_n : uf, second);
    flux += qy_n * us_n - qy_s * us_s;
    // [4] momentum and pressure (the fast build multiplies by one reciprocal of the span, which the compiler hoists
    // out of the tile's loop)
    const float abar = HALF * (h_l + h_r) * dx;
    // the face's momentum (the last step's abar * u, rounded once as that step rounded it)
    const float* HO = sm + L::HO;
    auto momentum = [&]() {
        return mst ? sm[L::M + AX * L::S + sl] : __fmul_rn(HALF * (HO[b - S] + HO[b]) * dx, uf);
    };
#ifdef W2B_FAST
    const float rspan = rcp_approx(span);
    const float press = dt * P.g * d_eta * rspan;
    float us;
    if (abar > 1e-6f * dx)
        us = qdiv(momentum() - dt * flux * rspan, abar) - press;
    else
        us = uf - press;
#else
    const float press = qdiv(dt * P.g * d_eta, span);
    float us;
    if (abar > 1e-6f * dx)
        us = qdiv(momentum() - qdiv(dt * flux, span), abar) - press;
    else
        us = uf - press;
#endif
    const float vb = 0.25f * (VP[b - S] + VP[b] + VP[b - S + PP] + VP[b + PP]);

    // the table lookup from the quad loaded in part A (common.cuh face_lookup); rowc holds, per row r, c0^2 and
    // c1^2 - c0^2 with c0 = r / m, c1 = (r + 1) / m, and in its last slot 1 - c^2 with c = (m - 1) / m: the very
    // float32 values the lookup forms, computed once a CTA
    const float top = st[4 * L::S + sl], e = F.eface;
    const float4 q = F.q;
    float area, tt, w;
    if (F.bits & FA_ABOVE) {
        const float a1 = q.z, a0 = q.x;
        w = qdiv(a1 - a0, top * rowc[2 * (A.rows - 1)]);
        area = a1 + w * (e - top);
        tt = q.w * qdiv(area, qmax(a1, 1e-12f));
    } else {
        const int r = F.bits & FA_ROW;
        const float e0 = rowc[2 * r] * top;
        const float de = rowc[2 * r + 1] * top;
#ifdef W2B_FAST
        const float rde = rcp_approx(de);  // one reciprocal for both quotients
        const float f = (e - e0) * rde;
        area = q.x + f * (q.z - q.x);
        tt = q.y + f * (q.w - q.y);
        w = (q.z - q.x) * rde;
#else
        const float f = qdiv(e - e0, de);
        area = q.x + f * (q.z - q.x);
        tt = q.y + f * (q.w - q.y);
        w = qdiv(q.z - q.x, de);
#endif
    }
    // [1] the volume-limited section
    float rho = ONE;
    if (ON || P.sheet) {
        const float avol = hup * dx;
        if (avol < area) {
            const float sub = qdiv(qmin(I.e_lp, I.e_rp), qmax(I.e_lp, I.e_rp));
            const float sub2 = sub * sub;
            const float alpha = sub2 * sub2;
            rho = alpha + qdiv((ONE - alpha) * avol, area);
        }
    }
    // [5] friction. The fast build forms 1 / max(tt^(10/3), 1e-30) and 1 / max(rho^(4/3), 1e-12) as capped powers from
    // the hardware log2 and exp2 (within about 1e-6 relative; tt = 0 or rho = 0 gives the cap, as the clamps do).
#ifdef W2B_FAST
    float fric = area * area * qmin(ex2_approx(-3.33333325f * lg2_approx(tt)), 1e30f);
    if (rho < ONE) fric = fric * qmin(ex2_approx(-1.33333337f * lg2_approx(rho)), 1e12f);
#else
    const float t3 = tt * tt * tt * qcbrt(tt);
    float fric = qdiv(area * area, qmax(t3, 1e-30f));
    if (rho < ONE) fric = qdiv(fric, qmax(rho * qcbrt(rho), 1e-12f));
#endif
    const float a = dt * P.g * fric;
    const float sp = qsqrt(us * us + vb * vb);
    float un = qdiv(2.0f * us, ONE + qsqrt(ONE + 4.0f * a * sp));
    if (fabsf(un) > P.u_max) un = un > ZERO ? P.u_max : -P.u_max;
    // [6] crest face
    float qn = area * rho * un;
    float c = st[5 * L::S + sl];
    if (c != ZERO) {
        float area_c = area, w_c = w;
        if (c < ZERO) {
            c = -c;
            const float ua = from_left ? um : up;
            float tc;
            const float4* quads = A.ftab4[AX] + (size_t)t * (A.rows - 1) * TILE2 + local;
            face_lookup(eup + qdiv(HALF * ua * ua, P.g), top, quads, A.rows, area_c, tc, w_c);
        }
        const float qc = c * area_c * qsqrt(qdiv(area_c, qmax(w_c, 1e-9f)));
        if (fabsf(qn) > qc) {
            qn = qn > ZERO ? qc : -qc;
            un = qdiv(qn, qmax(area * rho, 1e-12f));
        }
    }
    if constexpr (PROBE) {
        probe_un[local] = un;
    } else {
        A.uu[AX][1 - p][k] = un;
        A.q1[AX][k] = qn;
    }
    if (!want_wave) return ZERO;
    if (not_finite(un)) return 1e30f;
    const float* D = sm + L::off(F_D);
    const float d_left = D[b - S], d_right = D[b];
    const float dup = from_left ? d_left : d_right;
    if (dup <= P.h_cfl) return ZERO;
    // the plan shares of the face's two cells: from the image, or (a strip) from global memory at native index k
    float om_l, om_r;
    if constexpr (L::OM) {
        const float* OM = sm + L::off(F_OM);
        om_l = OM[b - S];
        om_r = OM[b];
    } else {
        om_l = A.om[k - (AX == 0 ? 1 : A.px)];
        om_r = A.om[k];
    }
    float plan = from_left ? om_l : om_r;
    const float dother = from_left ? d_right : d_left;
    if (dother > P.h_cfl) plan = qmin(plan, from_left ? om_r : om_l);
    const float wave = qsqrt(qmax(qdiv(P.g * area * rho, qmax(plan, P.a_min) * dx), ZERO));
    return fabsf(un) + qmin(P.lead * fabsf(un - uf), 2.0f * wave) + wave;
}

__device__ __forceinline__ float warp_max(float v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax32(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide max of v; the result is valid in thread 0. red holds one entry a warp.
__device__ __forceinline__ float block_max(float v, float* red) {
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int nw = (int)(blockDim.x * blockDim.y) / 32;
    v = warp_max(v);
    if ((tid & 31) == 0) red[tid >> 5] = v;
    __syncthreads();
    float r = 0.0f;
    if (tid < 32) {
        r = tid < nw ? red[tid] : 0.0f;
        r = warp_max(r);
    }
    __syncthreads();
    return r;
}

// The face pass: both own faces of every cell of the tiles of the work list (wadi2d/solver/gpu/kernels/faces.cu:
// 148-175). Each CTA (16 warps, a warp a tile row, two rows a warp; two CTAs a SM) stages a tile with TMA: nine
// 40 x 36 state boxes, the two momenta (or, once a face pass has stepped, the last step's mean depth box they are
// formed from), and the tile's twelve static face scalars as bulk copies; on refresh steps
// the tile's wave maximum goes to its run's maximum (an integer atomic max on the float bits). p is the parity of
// the run's ping-pong halves.
template <bool ON>
__global__ void __launch_bounds__(FACES_THREADS, 2) faces_kernel(const __grid_constant__ TMaps M, StepArgs A) {
    extern __shared__ __align__(128) float sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ float red[32];
    __shared__ float rowc[2 * 64 + 1];
    Ctl* ctl = A.ctl;
    if (!(ctl->any & ANY_RUN)) return;
    const int nwork = ctl->nwork;
    const int mst = ctl->m_stored;
    const int tid = threadIdx.x;
    if (tid == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
    }
    if (tid < A.rows - 1) {
        const float m = (float)(A.rows - 1);
        const float c0 = (float)tid / m;
        const float c1 = (float)(tid + 1) / m;
        rowc[2 * tid] = c0 * c0;
        rowc[2 * tid + 1] = c1 * c1 - c0 * c0;
    } else if (tid == A.rows - 1) {
        const float m = (float)(A.rows - 1);
        const float c = (m - 1.0f) / m;
        rowc[2 * tid] = 1.0f - c * c;
    }
    __syncthreads();
    const float* statics[12] = {A.fl[0], A.fr[0], A.gl[0], A.gr[0], A.ef[0], A.cw[0],
                                A.fl[1], A.fr[1], A.gl[1], A.gr[1], A.ef[1], A.cw[1]};
    uint32_t phase = 0;
    const int lane = tid & 31, warp = tid >> 5;
    for (int a = blockIdx.x; a < nwork; a += gridDim.x) {
        const int t = A.list[a];
        const int run = A.tile_run[t];
        const int flags = A.R.flags[run];
        if (!(flags & F_RUN)) continue;  // the tile's run has finished: uniform over the CTA
        const float dt = A.R.dtf[run];
        const float dx = A.R.dx[run];
        const int want_wave = (flags & F_WAVE) != 0;
        const int p = A.R.parity[run];
        const int tj = A.tiles[2 * t], ti = A.tiles[2 * t + 1];
        const int ts = table_of(A, t);
        if (tid == 0) {
            fence_proxy_async();
            mbar_expect_tx(&bar, (uint32_t)((NBOX - (want_wave ? 0 : 1)) * BOX + (mst ? 14 * TILE2 : BOX + 12 * TILE2)) * 4u);
            const int x0 = ti * TILE + GX - 4, y0 = tj * TILE + GY - 2;
            tma_load_2d(sm + F_D * BOX, &M.d, x0, y0, &bar);
            tma_load_2d(sm + F_H * BOX, &M.h[p], x0, y0, &bar);
            tma_load_2d(sm + F_U * BOX, &M.u[p], x0, y0, &bar);
            tma_load_2d(sm + F_V * BOX, &M.v[p], x0, y0, &bar);
            tma_load_2d(sm + F_QX * BOX, &M.qx, x0, y0, &bar);
            tma_load_2d(sm + F_QY * BOX, &M.qy, x0, y0, &bar);
            if (want_wave) tma_load_2d(sm + F_OM * BOX, &M.om, x0, y0, &bar);
            tma_load_2d(sm + F_ZCX * BOX, &M.zcx, x0, y0, &bar);
            tma_load_2d(sm + F_ZCY * BOX, &M.zcy, x0, y0, &bar);
            if (mst) {
                tma_load_2d(sm + SM_M, &M.mx[p], x0 + 4, y0 + 2, &bar);
                tma_load_2d(sm + SM_M + TILE2, &M.my[p], x0 + 4, y0 + 2, &bar);
            } else {
                tma_load_2d(sm + TileImage::HO, &M.h[1 - p], x0, y0, &bar);
            }
            for (int f = 0; f < 12; ++f) bulk_load(sm + SM_ST + f * TILE2, statics[f] + (size_t)ts * TILE2, TILE2 * 4, &bar);
        }
        const bool ok = mbar_wait(&bar, phase);
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
            // the copies did not land: report, give them one more bounded wait, and leave the loop
            if (tid == 0) atomicExch(&ctl->status, W2B_ETIMEOUT);
            mbar_wait(&bar, phase ^ 1u);
            return;
        }
        const int base = (tj * TILE + GY) * A.px + ti * TILE + GX;
        float wmax = 0.0f;
#pragma unroll 1
        for (int c = 0; c < 2; ++c) {
            const int jj = warp + 16 * c, ii = lane;
            const int local = jj * TILE + ii;
            const int b = (jj + 2) * BOXW + ii + 4;
            const int k = base + jj * A.px + ii;
            FaceA fx, fy;
            face_a<0, ON>(sm, b, local, local, A, ts, fx);
            face_a<1, ON>(sm, b, local, local, A, ts, fy);
            const float wx = face_bc<0, false, ON>(sm, b, local, local, k, A, ts, fx, dt, dx, want_wave, rowc, p, mst);
            const float wy = face_bc<1, false, ON>(sm, b, local, local, k, A, ts, fy, dt, dx, want_wave, rowc, p, mst);
            wmax = fmax32(wmax, fmax32(wx, wy));
        }
        if (want_wave) {
            // the tile's wave, and the run's maximum (wadi2d/solver/gpu/kernels/common.cuh:93-96: positive floats
            // order like their bit patterns, so the integer maximum is the float maximum)
            const float bm = block_max(wmax, red);
            if (tid == 0) {
                A.wave[t] = bm;
                atomicMax(A.R.wave_bits + run, __float_as_uint(bm));
            }
        } else {
            __syncthreads();
        }
    }
}

// The wave speed and the new velocity of every own face of tile t for a step dt from the current state, as the face
// pass would compute them, written to out ([wx | wy | un_x | un_y], 1024 each, tile layout) and nothing else: the
// device side of the step limiter (wadi2d/solver/limiter.py:31-55, the CPU twin's face_step on one tile). One CTA;
// the tile's image is filled with plain loads (the boxes lie inside the guard ring of the NATIVE arrays).
__global__ void __launch_bounds__(1024) probe_kernel(StepArgs A, int t, float dt, float* __restrict__ out) {
    extern __shared__ __align__(128) float sm[];
    __shared__ float rowc[2 * 64 + 1];
    const int tid = threadIdx.x;
    const int run = A.tile_run[t];
    const int p = A.R.parity[run];
    const float dx = A.R.dx[run];
    const int tj = A.tiles[2 * t], ti = A.tiles[2 * t + 1];
    const int x0 = ti * TILE + GX - 4, y0 = tj * TILE + GY - 2;
    const int mst = A.ctl->m_stored;
    const float* boxes[NBOX] = {A.d, A.hh[p], A.uu[0][p], A.uu[1][p], A.q[0], A.q[1], A.om, A.zc[0], A.zc[1]};
    for (int idx = tid; idx < BOX; idx += blockDim.x) {
        const size_t k = (size_t)(y0 + idx / BOXW) * A.px + x0 + idx % BOXW;
        for (int f = 0; f < NBOX; ++f) sm[f * BOX + idx] = boxes[f][k];
        if (!mst) sm[TileImage::HO + idx] = A.hh[1 - p][k];
    }
    const float* statics[12] = {A.fl[0], A.fr[0], A.gl[0], A.gr[0], A.ef[0], A.cw[0],
                                A.fl[1], A.fr[1], A.gl[1], A.gr[1], A.ef[1], A.cw[1]};
    for (int idx = tid; idx < TILE2; idx += blockDim.x) {
        const size_t k = (size_t)(tj * TILE + GY + idx / TILE) * A.px + ti * TILE + GX + idx % TILE;
        if (mst) {
            sm[SM_M + idx] = A.mm[0][p][k];
            sm[SM_M + TILE2 + idx] = A.mm[1][p][k];
        }
        for (int f = 0; f < 12; ++f) sm[SM_ST + f * TILE2 + idx] = statics[f][(size_t)table_of(A, t) * TILE2 + idx];
    }
    if (tid < A.rows - 1) {
        const float m = (float)(A.rows - 1);
        const float c0 = (float)tid / m;
        const float c1 = (float)(tid + 1) / m;
        rowc[2 * tid] = c0 * c0;
        rowc[2 * tid + 1] = c1 * c1 - c0 * c0;
    } else if (tid == A.rows - 1) {
        const float m = (float)(A.rows - 1);
        const float c = (m - 1.0f) / m;
        rowc[2 * tid] = 1.0f - c * c;
    }
    __syncthreads();
    const int jj = tid >> 5, ii = tid & 31;
    const int local = jj * TILE + ii;
    const int b = (jj + 2) * BOXW + ii + 4;
    const int k = (tj * TILE + GY + jj) * A.px + ti * TILE + GX + ii;
    FaceA fx, fy;
    const int ts = table_of(A, t);
    face_a<0>(sm, b, local, local, A, ts, fx);
    face_a<1>(sm, b, local, local, A, ts, fy);
    out[local] = face_bc<0, true>(sm, b, local, local, k, A, ts, fx, dt, dx, 1, rowc, p, mst, out + 2 * TILE2);
    out[TILE2 + local] = face_bc<1, true>(sm, b, local, local, k, A, ts, fy, dt, dx, 1, rowc, p, mst, out + 3 * TILE2);
}

void launch_probe(const StepArgs& A, int t, float dt, float* out, cudaStream_t s) {
    probe_kernel<<<1, 1024, SM_FLOATS * 4, s>>>(A, t, dt, out);
}

// The strip forms of the face pass: the same faces, a strip of H rows of a tile at a time (H = 16: halves, H = 8:
// quarters). A unit of work is one strip of a tile of the work list (32 / H units a tile); a CTA of 16 H threads (H / 2
// warps, two rows a warp) stages the strip with TMA as eight 40-column boxes of the rows each state field is read at
// (StripImage), its momenta as 32 x H boxes and its twelve static face scalars as bulk copies: 51 KB for 16 rows, so
// that four CTAs share a SM, 27 KB for 8 rows, eight (with 64 registers a thread). While one CTA waits for its copies
// the others compute (the tile form's two CTAs of 109 KB leave a SM idle whenever both wait). The plan shares, wanted
// on refresh steps only, are read from
// global memory. A face's arithmetic is the tile form's, bit for bit. On refresh steps each strip's wave maximum goes
// to its tile's entry and its run's maximum by integer atomic maxima on the float bits.
template <int H, bool ON>
__global__ void __launch_bounds__(StripImage<H>::THREADS, StripImage<H>::CTAS)
    strips_kernel(const __grid_constant__ TMaps M, StepArgs A) {
    using L = StripImage<H>;
    constexpr int PER = TILE / H;  // strips a tile
    const StripMaps& SM_ = H == 16 ? M.s16 : M.s8;
    extern __shared__ __align__(128) float sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ float red[L::THREADS / 32];
    __shared__ float rowc[2 * 64 + 1];
    Ctl* ctl = A.ctl;
    if (!(ctl->any & ANY_RUN)) return;
    const int nunits = PER * ctl->nwork;
    const int mst = ctl->m_stored;
    const int tid = threadIdx.x;
    if (tid == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
    }
    if (tid < A.rows - 1) {
        const float m = (float)(A.rows - 1);
        const float c0 = (float)tid / m;
        const float c1 = (float)(tid + 1) / m;
        rowc[2 * tid] = c0 * c0;
        rowc[2 * tid + 1] = c1 * c1 - c0 * c0;
    } else if (tid == A.rows - 1) {
        const float m = (float)(A.rows - 1);
        const float c = (m - 1.0f) / m;
        rowc[2 * tid] = 1.0f - c * c;
    }
    __syncthreads();
    const float* statics[12] = {A.fl[0], A.fr[0], A.gl[0], A.gr[0], A.ef[0], A.cw[0],
                                A.fl[1], A.fr[1], A.gl[1], A.gr[1], A.ef[1], A.cw[1]};
    uint32_t phase = 0;
    const int lane = tid & 31, warp = tid >> 5;
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const int t = A.list[u / PER];
        const int row0 = (u % PER) * H;
        const int run = A.tile_run[t];
        const int flags = A.R.flags[run];
        if (!(flags & F_RUN)) continue;  // the tile's run has finished: uniform over the CTA
        const float dt = A.R.dtf[run];
        const float dx = A.R.dx[run];
        const int want_wave = (flags & F_WAVE) != 0;
        const int p = A.R.parity[run];
        const int tj = A.tiles[2 * t], ti = A.tiles[2 * t + 1];
        const int ts = table_of(A, t);
        if (tid == 0) {
            fence_proxy_async();
            mbar_expect_tx(&bar, (uint32_t)(mst ? L::BYTES : L::BYTES_HO));
            // each box from its first row (the strip's row 0 is y)
            const int x0 = ti * TILE + GX - 4, y = tj * TILE + GY + row0;
            tma_load_2d(sm + L::S_U, &SM_.u[p], x0, y - 2, &bar);
            tma_load_2d(sm + L::S_V, &SM_.v[p], x0, y - 2, &bar);
            tma_load_2d(sm + L::S_D, &SM_.d, x0, y - 1, &bar);
            tma_load_2d(sm + L::S_H, &SM_.h[p], x0, y - 1, &bar);
            tma_load_2d(sm + L::S_QX, &SM_.qx, x0, y - 1, &bar);
            tma_load_2d(sm + L::S_QY, &SM_.qy, x0, y - 1, &bar);
            tma_load_2d(sm + L::S_ZCX, &SM_.zcx, x0, y, &bar);
            tma_load_2d(sm + L::S_ZCY, &SM_.zcy, x0, y - 1, &bar);
            if (mst) {
                tma_load_2d(sm + L::M, &SM_.mx[p], x0 + 4, y, &bar);
                tma_load_2d(sm + L::M + L::S, &SM_.my[p], x0 + 4, y, &bar);
            } else {
                tma_load_2d(sm + L::M, &SM_.h[1 - p], x0, y - 1, &bar);  // the mean depth box's rows
            }
            for (int f = 0; f < 12; ++f)
                bulk_load(sm + L::ST + f * L::S, statics[f] + (size_t)ts * TILE2 + row0 * TILE, L::S * 4, &bar);
        }
        const bool ok = mbar_wait(&bar, phase);
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
            // the copies did not land: report, give them one more bounded wait, and leave the loop
            if (tid == 0) atomicExch(&ctl->status, W2B_ETIMEOUT);
            mbar_wait(&bar, phase ^ 1u);
            return;
        }
        const int base = (tj * TILE + GY) * A.px + ti * TILE + GX;
        float wmax = 0.0f;
#pragma unroll 1
        for (int c = 0; c < 2; ++c) {
            const int js = warp + (H / 2) * c, ii = lane;  // the row in the strip, and in the tile
            const int jj = row0 + js;
            const int sl = js * TILE + ii, local = jj * TILE + ii;
            const int b = (js + 2) * BOXW + ii + 4;
            const int k = base + jj * A.px + ii;
            FaceA fx, fy;
            face_a<0, ON, L>(sm, b, sl, local, A, ts, fx);
            face_a<1, ON, L>(sm, b, sl, local, A, ts, fy);
            const float wx = face_bc<0, false, ON, L>(sm, b, sl, local, k, A, ts, fx, dt, dx, want_wave, rowc,
                                                               p, mst);
            const float wy = face_bc<1, false, ON, L>(sm, b, sl, local, k, A, ts, fy, dt, dx, want_wave, rowc,
                                                               p, mst);
            wmax = fmax32(wmax, fmax32(wx, wy));
        }
        if (want_wave) {
            const float bm = block_max(wmax, red);
            if (tid == 0) {
                atomicMax(reinterpret_cast<unsigned int*>(A.wave) + t, __float_as_uint(bm));
                atomicMax(A.R.wave_bits + run, __float_as_uint(bm));
            }
        } else {
            __syncthreads();
        }
    }
}

cudaError_t faces_setup() {
    cudaError_t e = cudaFuncSetAttribute(probe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SM_FLOATS * 4);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(faces_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                    FACES_SMEM);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(faces_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                    FACES_SMEM);
    for (auto k : {strips_kernel<16, true>, strips_kernel<16, false>}) {
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, StripImage<16>::SMEM);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    }
    for (auto k : {strips_kernel<8, true>, strips_kernel<8, false>}) {
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, StripImage<8>::SMEM);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    }
    return e;
}

// The resident CTAs a SM of the strip form of `rows` rows (16 or 8).
int strips_occupancy(int rows) {
    int on = 0, off = 0;
    if (rows == 16) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&on, strips_kernel<16, true>, StripImage<16>::THREADS,
                                                      StripImage<16>::SMEM);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&off, strips_kernel<16, false>, StripImage<16>::THREADS,
                                                      StripImage<16>::SMEM);
    } else {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&on, strips_kernel<8, true>, StripImage<8>::THREADS,
                                                      StripImage<8>::SMEM);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&off, strips_kernel<8, false>, StripImage<8>::THREADS,
                                                      StripImage<8>::SMEM);
    }
    return on < off ? on : off;
}

// The face pass in its strip form of `rows` rows (16 or 8); grid: CTAs (the units are the work list's tiles, 32 /
// rows strips each).
void launch_strips(int rows, const TMaps& M, const StepArgs& A, int grid, cudaStream_t s) {
    const bool on = A.P.second && A.P.sheet && A.P.mirror && A.P.carry;
    if (rows == 16) {
        if (on)
            strips_kernel<16, true><<<grid, StripImage<16>::THREADS, StripImage<16>::SMEM, s>>>(M, A);
        else
            strips_kernel<16, false><<<grid, StripImage<16>::THREADS, StripImage<16>::SMEM, s>>>(M, A);
    } else {
        if (on)
            strips_kernel<8, true><<<grid, StripImage<8>::THREADS, StripImage<8>::SMEM, s>>>(M, A);
        else
            strips_kernel<8, false><<<grid, StripImage<8>::THREADS, StripImage<8>::SMEM, s>>>(M, A);
    }
}

// The resident CTAs a SM of the face pass (the smaller of its two forms').
int faces_occupancy() {
    int on = 0, off = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&on, faces_kernel<true>, FACES_THREADS, FACES_SMEM);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&off, faces_kernel<false>, FACES_THREADS, FACES_SMEM);
    return on < off ? on : off;
}

// The face pass, in its form with the numerics switches folded in when they are all on (the reference's defaults).
void launch_faces(const TMaps& M, const StepArgs& A, int grid, cudaStream_t s) {
    if (A.P.second && A.P.sheet && A.P.mirror && A.P.carry)
        faces_kernel<true><<<grid, FACES_THREADS, FACES_SMEM, s>>>(M, A);
    else
        faces_kernel<false><<<grid, FACES_THREADS, FACES_SMEM, s>>>(M, A);
}

// ------------------------------------------------------------------ update pass

__device__ __forceinline__ float scaled(float q, float rl, float rr) { return q * (q > 0.0f ? rl : rr); }

constexpr int RING = TILE + 2;  // the tile and its one-cell ring
constexpr int RPAD = RING + 1;
constexpr int U_QX1 = 0, U_QY1 = 1, U_H = 2;       // 40 x 36 boxes
constexpr int U_OWN = 3 * BOX;                      // res, src, hc: 32 x 32 each
constexpr int U_R = U_OWN + 3 * TILE2;              // r of the tile and its ring
constexpr int U_LP = (U_R + RING * RPAD + 31) / 32 * 32;  // the tile's cached level pairs (float2), 128-byte aligned
constexpr int U_LR = U_LP + 2 * TILE2;                     // and their rows (bytes)
constexpr int U_FLOATS = U_LR + TILE2 / 4;
constexpr int UPDATE_SMEM = U_FLOATS * 4;           // 43,648 bytes: four CTAs a SM
static_assert(UPDATE_SMEM == 43648, "update image size");
constexpr int UPDATE_THREADS = 256;

// The first entry at or after a, in steps of the grid, whose run is stepping (the same for every thread of a CTA).
__device__ __forceinline__ int next_tile(const StepArgs& A, int a, int nwork) {
    for (; a < nwork; a += gridDim.x)
        if (A.R.flags[A.tile_run[A.list[a]]] & F_RUN) break;
    return a;
}

// Issue (thread 0) the copies of tile t's update image against bar: the unscaled discharges and the old depth with
// their ring, the residual, the source and Hc, and the tile's level cache (each cell's last level pair and its row).
__device__ __forceinline__ void update_issue(float* sm, uint64_t* bar, const TMaps& M, const StepArgs& A, int t) {
    const int p = A.R.parity[A.tile_run[t]];
    const int tj = A.tiles[2 * t], ti = A.tiles[2 * t + 1];
    fence_proxy_async();
    mbar_expect_tx(bar, (uint32_t)(3 * BOX + 3 * TILE2) * 4u + (uint32_t)TILE2 * 9u);
    const int x0 = ti * TILE + GX - 4, y0 = tj * TILE + GY - 2;
    tma_load_2d(sm + U_QX1 * BOX, &M.qx1, x0, y0, bar);
    tma_load_2d(sm + U_QY1 * BOX, &M.qy1, x0, y0, bar);
    tma_load_2d(sm + U_H * BOX, &M.h[p], x0, y0, bar);
    tma_load_2d(sm + U_OWN, &M.res, x0 + 4, y0 + 2, bar);
    tma_load_2d(sm + U_OWN + TILE2, &M.src, x0 + 4, y0 + 2, bar);
    bulk_load(sm + U_OWN + 2 * TILE2, A.hc + (size_t)table_of(A, t) * TILE2, TILE2 * 4, bar);
    bulk_load(sm + U_LP, A.lpair + (size_t)t * TILE2, TILE2 * 8, bar);
    bulk_load(sm + U_LR, A.lrow + (size_t)t * TILE2, TILE2, bar);
}

// The update pass (wadi2d/solver/gpu/kernels/cells.cu:4-63 with limit fused in): TMA stages the tile's unscaled
// discharges and old depth with their ring, its residual, source and Hc, and its level cache; r of the tile and its
// one-cell ring is formed in shared memory; then each thread takes its four cells through continuity and takes their
// level pairs from the cache, or for the cells whose row changed from the table (the gathers issued together). Once
// every thread has read the image, thread 0 issues the next tile's copies into it, and they land while any gathers
// return and the level, the wet share and the wet flag are finished.
__global__ void __launch_bounds__(UPDATE_THREADS) update_kernel(const __grid_constant__ TMaps M, StepArgs A) {
    extern __shared__ __align__(128) float sm[];
    __shared__ __align__(8) uint64_t bar;
    Ctl* ctl = A.ctl;
    if (!(ctl->any & ANY_RUN)) return;
    const int nwork = ctl->nwork;
    const int px = A.px;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    // the face pass before this one has stepped: from now on the momenta are formed from the state (Ctl::m_stored)
    if (blockIdx.x == 0 && tid == 0) ctl->m_stored = 0;
    const int rows = A.rows, last = rows - 1;
    if (tid == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
    }
    __syncthreads();
    uint32_t phase = 0;
    const float* QX1 = sm + U_QX1 * BOX;
    const float* QY1 = sm + U_QY1 * BOX;
    const float* H = sm + U_H * BOX;
    const float* RES = sm + U_OWN;
    const float* SRC = sm + U_OWN + TILE2;
    const float* HC = sm + U_OWN + 2 * TILE2;
    float* rs = sm + U_R;
    int a = next_tile(A, blockIdx.x, nwork);
    if (tid == 0 && a < nwork) update_issue(sm, &bar, M, A, A.list[a]);
    while (a < nwork) {
        const int t = A.list[a];
        const int run = A.tile_run[t];
        const int flags = A.R.flags[run];
        const float dt = A.R.dtf[run];
        const float dxr = A.R.dx[run];
        const float area = dxr * dxr;
        const int want_plan = (flags & F_WAVE) != 0;
        const int want_wet = (flags & F_WET) != 0;
        const int p = A.R.parity[run];
        float* __restrict__ h_next = A.hh[1 - p];
        const int tj = A.tiles[2 * t], ti = A.tiles[2 * t + 1];
        const bool ok = mbar_wait(&bar, phase);
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicExch(&ctl->status, W2B_ETIMEOUT);
            mbar_wait(&bar, phase ^ 1u);
            return;
        }
        // positivity ratio r (wadi2d/solver/gpu/kernels/cells.cu:4-19) of the tile and its ring, from the old h
        for (int idx = tid; idx < RING * RING; idx += UPDATE_THREADS) {
            const int rj = idx / RING, ri = idx - rj * RING;
            const int b = (rj + 1) * BOXW + ri + 3;  // cell (rj - 1, ri - 1)
            const float out = fmax32(QX1[b + 1], 0.0f) + fmax32(-QX1[b], 0.0f) + fmax32(QY1[b + BOXW], 0.0f) +
                              fmax32(-QY1[b], 0.0f);
            const float have = fmax32(H[b], 0.0f) * area;
            rs[rj * RPAD + ri] = out * dt > have ? have / (out * dt) : 1.0f;
        }
        __syncthreads();
        const int base = (tj * TILE + GY) * px + ti * TILE + GX;
        const float2* __restrict__ pairs_t = A.dtab2 + (size_t)table_of(A, t) * (rows - 1) * TILE2;
        // continuity (cells.cu:219-232) for the thread's four cells
        float hn[4], sv[4], hcs[4];
        int rr[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int jj = threadIdx.y * 4 + c, ii = threadIdx.x;
            const int local = jj * TILE + ii;
            const int b = (jj + 2) * BOXW + ii + 4;
            const int k = base + jj * px + ii;
            const float* row = rs + (jj + 1) * RPAD + (ii + 1);
            const float rc = row[0];
            const float qw = scaled(QX1[b], row[-1], rc);
            const float qe = scaled(QX1[b + 1], rc, row[1]);
            const float qn = scaled(QY1[b], row[-RPAD], rc);
            const float qs = scaled(QY1[b + BOXW], rc, row[RPAD]);
            A.q[0][k] = qw;
            A.q[1][k] = qn;
            const float h0 = H[b];
            const float inc = RES[local] + dt * SRC[local] - dt * (qe - qw + qs - qn) / area;
            const float total = h0 + inc;
            hn[c] = fmax32(total, 0.0f);
            A.res[k] = total > 0.0f ? inc - (total - h0) : 0.0f;
            h_next[k] = hn[c];
            // the level table's row (common.cuh cell_level): the top row above Hc, none where Hc <= 0
            const float hcv = HC[local];
            hcs[c] = hcv;
            if (hcv <= 0.0f) {
                rr[c] = -1;
                sv[c] = 0.0f;
            } else if (hn[c] >= hcv) {
                rr[c] = last - 1;
                sv[c] = -1.0f;
            } else {
                sv[c] = sqrtf(hn[c] / hcv) * (float)last;
                rr[c] = row_of(sv[c], last);
            }
        }
        // the level pairs: the cached one where the cell's row is the cached row (about 699 cells in 700 from one
        // step to the next), else gathered from the table and cached
        float2 pr[4];
        const float2* LP = reinterpret_cast<const float2*>(sm + U_LP);
        const uint8_t* LR = reinterpret_cast<const uint8_t*>(sm + U_LR);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int local = (threadIdx.y * 4 + c) * TILE + threadIdx.x;
            if (rr[c] < 0) {
                pr[c] = make_float2(0.0f, 0.0f);
            } else if (LR[local] == rr[c]) {
                pr[c] = LP[local];
            } else {
                pr[c] = __ldg(pairs_t + (size_t)rr[c] * TILE2 + local);
                A.lpair[(size_t)t * TILE2 + local] = pr[c];
                A.lrow[(size_t)t * TILE2 + local] = (uint8_t)rr[c];
            }
        }
        // every thread has read the image and r: the next tile's copies land in it during this tile's gathers
        __syncthreads();
        const int an = next_tile(A, a + gridDim.x, nwork);
        if (tid == 0 && an < nwork) update_issue(sm, &bar, M, A, A.list[an]);
        int any = 0;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int jj = threadIdx.y * 4 + c, ii = threadIdx.x;
            const int k = base + jj * px + ii;
            const float hcv = hcs[c];
            const float h = hn[c];
            float dk, om = 1.0f;
            if (hcv <= 0.0f) {
                dk = h;
            } else if (h >= hcv) {
                dk = pr[c].y + (h - hcv);
            } else {
                const int r = rr[c];
                const float2 q = pr[c];
                if (A.P.level_fp64 && r == 0) {
                    const double sd = sqrt((double)h / (double)hcv) * (double)last;
                    dk = (float)((double)q.x + sd * ((double)q.y - (double)q.x));
                } else {
                    dk = q.x + (sv[c] - (float)r) * (q.y - q.x);
                }
                const float m = (float)last;
                om = hcv * (float)(2 * r + 1) / (m * m) / fmax32(q.y - q.x, 1e-12f);
            }
            A.d[k] = dk;
            if (want_plan) A.om[k] = om;
            any |= h > 0.0f;
        }
        if (want_wet) {
            const int w = __syncthreads_or(any);
            if (tid == 0) A.wet[t] = w;
        }
        a = an;
    }
}

cudaError_t update_setup() {
    return cudaFuncSetAttribute(update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, UPDATE_SMEM);
}

int update_occupancy() {
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, update_kernel, UPDATE_THREADS, UPDATE_SMEM);
    return occ;
}

void launch_update(const TMaps& M, const StepArgs& A, int grid, cudaStream_t s) {
    update_kernel<<<grid, dim3(32, 8), UPDATE_SMEM, s>>>(M, A);
}

}  // namespace W2B_ARITH

#ifndef W2B_FAST
// ------------------------------------------------------------------ self-checks

// Every positive float from first (as bits) on: cbrt32 against the double path; out[0] counts mismatches,
// out[1..4] keep some mismatching inputs.
__global__ void cbrt_check_kernel(uint32_t first, uint32_t count, unsigned long long* out) {
    for (uint64_t n = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; n < count; n += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t bits = first + (uint32_t)n;
        const float x = __uint_as_float(bits);
        const float a = cbrt32(x);
        const float b = (float)cbrt((double)x);
        if (__float_as_uint(a) != __float_as_uint(b) && !(isnan(a) && isnan(b))) {
            const unsigned long long k = atomicAdd(out, 1ull);
            if (k < 4) out[1 + k] = bits;
        }
    }
}

void launch_cbrt_check(uint32_t first, uint32_t count, unsigned long long* out, cudaStream_t s) {
    cbrt_check_kernel<<<148 * 16, 256, 0, s>>>(first, count, out);
}

// The bounded wait's give-up path, run on purpose: thread 0 arms a barrier for 16 bytes that no copy will bring, so
// its phase cannot complete, and waits on it with mbar_wait for `polls` polls. Nothing is in flight, so the CTA may
// leave. out[0] = W2B_ETIMEOUT if the wait gave up (W2B_OK if it completed, which it cannot), out[1] = the clock
// cycles the wait took.
__global__ void wait_check_kernel(uint32_t polls, long long* out) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    fence_barrier_init();
    mbar_expect_tx(&bar, 16);  // the one arrival, with 16 bytes still expected
    const long long t0 = clock64();
    const bool ok = mbar_wait(&bar, 0, polls);
    out[1] = clock64() - t0;
    out[0] = ok ? W2B_OK : W2B_ETIMEOUT;
}

void launch_wait_check(uint32_t polls, long long* out, cudaStream_t s) { wait_check_kernel<<<1, 32, 0, s>>>(polls, out); }

// ------------------------------------------------------------------ face momenta

// The face momenta into their arrays (each run's current half), as the face pass forms them once a face pass has
// stepped: the last step's abar * u, abar from the other half of the mean depth pair (the depths that step started
// from), rounded once. Every own face of every tile; nothing when the arrays already hold the momenta
// (Ctl::m_stored), so it may run before any read or write of the state. momentum_mark_kernel, after it, records that
// they do.
__global__ void momentum_kernel(StepArgs A) {
    if (A.ctl->m_stored) return;
    const long long n = (long long)(A.ntiles - 1) * TILE2;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int t = 1 + (int)(i / TILE2), c = (int)(i % TILE2);  // tile 0 is the void tile
        const int run = A.tile_run[t];
        const int p = A.R.parity[run];
        const float dx = A.R.dx[run];
        const int tj = A.tiles[2 * t], ti = A.tiles[2 * t + 1];
        const size_t k = (size_t)(tj * TILE + GY + c / TILE) * A.px + ti * TILE + GX + c % TILE;
        const float* ho = A.hh[1 - p];
        A.mm[0][p][k] = __fmul_rn(0.5f * (ho[k - 1] + ho[k]) * dx, A.uu[0][p][k]);
        A.mm[1][p][k] = __fmul_rn(0.5f * (ho[k - A.px] + ho[k]) * dx, A.uu[1][p][k]);
    }
}

__global__ void momentum_mark_kernel(Ctl* ctl) { ctl->m_stored = 1; }

void launch_momentum(const StepArgs& A, int sms, cudaStream_t s) {
    momentum_kernel<<<sms * 4, 256, 0, s>>>(A);
    momentum_mark_kernel<<<1, 1, 0, s>>>(A.ctl);
}

// ------------------------------------------------------------------ envelope pass

// The envelope of one own cell (wadi2d/engine/maxima.py:75-92; the CPU twin forms the centre speed in float64) with
// every load issued before any store, so that a thread's loads make one round trip; only the entries that change are
// written. un, vn: the face velocities after the step.
__device__ __forceinline__ void envelope_cell(const StepArgs& A, int fid, int k, float dk, float hk, float time,
                                              float arrive, float deep, const float* un, const float* vn) {
    const float d0 = A.env[0][fid], h0 = A.env[1][fid], s0 = A.env[2][fid], z0 = A.env[3][fid];
    const float a0 = A.env[4][fid];
    const float ue = un[k + 1], uw = un[k], vs = vn[k + A.px], vn0 = vn[k];
    // max(old, new) as fmax32 forms it keeps old exactly when old >= new
    if (!(d0 >= dk)) A.env[0][fid] = dk;
    if (!(h0 >= hk)) A.env[1][fid] = hk;
    if (dk > deep) {
        const double uc = 0.5 * (double)(uw + ue);
        const double vc = 0.5 * (double)(vn0 + vs);
        const double sp = sqrt(uc * uc + vc * vc);
        if (!((double)s0 >= sp)) A.env[2][fid] = (float)sp;
        const double hz = sp * (double)dk;
        if (!((double)z0 >= hz)) A.env[3][fid] = (float)hz;
    }
    if (a0 < 0.0f && dk >= arrive) A.env[4][fid] = time;
}

// The envelope after a step of the device loop, for the own cells of the work list's tiles whose runs record it at
// this step (F_MAX); boundary cells are recorded by the boundary pass after its overwrite. A CTA a tile at a time, a
// thread a cell; on steps that record no envelope every CTA returns at once.
// A tile's place (work list -> tile -> its run, its first own cell, its rows' boundary marks) is a chain of dependent
// loads, each from L2; the CTA stages it for ENV_CHUNK of its tiles at once in shared memory (all chains in flight
// together), so that a tile's own work waits on its run's flags (L1-resident) and then on its cells' data only.
constexpr int ENV_CHUNK = 64;
__global__ void __launch_bounds__(TILE2, 2) envelope_kernel(StepArgs A) {
    __shared__ int3 place[ENV_CHUNK];            // tile, run, native index of the tile's first own cell
    __shared__ uint32_t marks[ENV_CHUNK * TILE];  // the tile's boundary marks, a word a row
    Ctl* ctl = A.ctl;
    if (!(ctl->any & ANY_MAX)) return;
    const int nwork = ctl->nwork;
    const float arrive = ctl->arrive, deep = ctl->deep;
    const int tid = threadIdx.x, jj = tid >> 5, ii = tid & 31;
    const int G = gridDim.x;
    const int mine = (nwork - (int)blockIdx.x + G - 1) / G;  // this CTA's tiles: work positions blockIdx.x + i G
    for (int c0 = 0; c0 < mine; c0 += ENV_CHUNK) {
        const int nc = min(ENV_CHUNK, mine - c0);
        if (tid < nc) {
            const int t = A.list[blockIdx.x + (c0 + tid) * G];
            place[tid] = make_int3(t, A.tile_run[t],
                                   (A.tiles[2 * t] * TILE + GY) * A.px + A.tiles[2 * t + 1] * TILE + GX);
        }
        __syncthreads();
        for (int q = tid; q < nc * TILE; q += TILE2) marks[q] = A.bmark[place[q / TILE].x * TILE + q % TILE];
        __syncthreads();
        for (int i = 0; i < nc; ++i) {
            const int3 w = place[i];
            const int run = w.y;
            if ((A.R.flags[run] & (F_RUN | F_MAX)) != (F_RUN | F_MAX)) continue;
            if ((marks[i * TILE + jj] >> ii) & 1u) continue;
            const int p = A.R.parity[run];
            const int k = w.z + jj * A.px + ii;
            envelope_cell(A, w.x * TILE2 + tid, k, A.d[k], A.hh[1 - p][k], A.R.max_time[run], arrive, deep,
                          A.uu[0][1 - p], A.uu[1][1 - p]);
        }
        __syncthreads();  // the chunk's places and marks are read by every thread before the next chunk's overwrite
    }
}

// ------------------------------------------------------------------ boundary, tally, control (one CTA)

// Boundary cells of every running run (wadi2d/solver/gpu/kernels/cells.cu:95-111) and their envelope entries after
// the overwrite; in the device loop (control = 1) also the FP64 tally of every step and the design lines. Every item
// is independent of the others (a follow boundary reads an interior cell), so the kernel is a grid-stride loop over
// them: boundary cells, then tally faces, then one warp a line.
__global__ void boundary_kernel(StepArgs A, int control) {
    Ctl* ctl = A.ctl;
    if (!(ctl->any & ANY_RUN)) return;
    const RunTab& R = A.R;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gstride = gridDim.x * blockDim.x;
    for (int m = gtid; m < A.nb; m += gstride) {
        const int k = A.bcell[m];
        const int run = A.tile_run[tile_of_native(A, k)];
        const int flags = R.flags[run];
        if (!(flags & F_RUN)) continue;
        const int n = 1 - R.parity[run];
        float* h_next = A.hh[n];
        const int kind = A.bkind[m];
        if (kind == 0) {
            h_next[k] = A.bh0[m];
            A.d[k] = A.bd0[m];
        } else if (kind == 1) {
            h_next[k] = 0.0f;
            A.d[k] = 0.0f;
        } else {
            const int r = A.bref[m];
            h_next[k] = h_next[r];
            A.d[k] = fmax32(A.d[r] + A.bd0[m], 0.0f);
        }
        if ((flags & F_MAX) == F_MAX)
            envelope_cell(A, fid_of_native(A, k), k, A.d[k], h_next[k], R.max_time[run], ctl->arrive, ctl->deep,
                          A.uu[0][n], A.uu[1][n]);
    }
    if (!control) return;
    for (int m = gtid; m < A.ntally; m += gstride) {
        const int face = A.tface[m];
        const int run = A.tile_run[tile_of_native(A, face)];
        if (!(R.flags[run] & F_RUN)) continue;
        const float qv = A.taxis[m] ? A.q[1][face] : A.q[0][face];
        A.ttotal[m] += R.dt_tally[run] * (double)(A.tsign[m] * qv);
    }
    // design lines (wadi2d/engine/monitor.py:229-232 at every step): Q = sum of sign q over the line's faces, FP64,
    // lane-strided then a fixed shuffle tree; the running peak of |Q| and the time at the end of the step
    const int lane = threadIdx.x & 31;
    const int gwarp = gtid >> 5, nwarps = gstride >> 5;
    for (int l = gwarp; l < A.nlines; l += nwarps) {
        const int s = A.lstart[l], e = A.lstart[l + 1];
        if (s >= e) continue;
        const int run = A.tile_run[tile_of_native(A, A.lface[s])];
        if (!(R.flags[run] & F_RUN)) continue;
        double acc = 0.0;
        for (int m = s + lane; m < e; m += 32) {
            const int f = A.lface[m];
            acc += (double)A.lsign[m] * (double)(A.laxis[m] ? A.q[1][f] : A.q[0][f]);
        }
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
        if (lane == 0) {
            A.lq[l] = acc;
            const double a = fabs(acc);
            if (a > A.lpeak[l]) {
                A.lpeak[l] = a;
                A.ltime[l] = R.t[run] + R.dt_step[run];
            }
        }
    }
}

// Each running run's clock after its step (wadi2d/solver/stepper.py:113-124): the swap of its halves, t, the step
// counts, the step rule on refresh steps (dt_min and non-finite checks); a run that stops marks the work list for
// rebuilding. The threads of one CTA, after boundary_kernel.
__device__ void run_clocks(const StepArgs& A) {
    Ctl* ctl = A.ctl;
    if (!(ctl->any & ANY_RUN)) return;
    const RunTab& R = A.R;
    for (int r = threadIdx.x; r < A.nruns; r += blockDim.x) {
        if (!(R.flags[r] & F_RUN)) continue;
        R.parity[r] ^= 1;
        R.t[r] = R.t[r] + R.dt_step[r];
        R.nsteps[r] += 1;
        R.steps_run[r] += 1;
        if (R.flags[r] & F_WAVE) {
            R.wave_last[r] = __uint_as_float(R.wave_bits[r]);
            const double w = (double)__uint_as_float(R.wave_bits[r]);
            if (!isfinite(w)) {
                R.status[r] = W2B_ENONFINITE;
            } else {
                const double lim = ctl->cfl * (double)R.dx[r] / (ctl->wave_floor > w ? ctl->wave_floor : w);
                R.dt[r] = ctl->dt_max < lim ? ctl->dt_max : lim;
                if (R.dt[r] < ctl->dt_min) R.status[r] = W2B_EDTMIN;
            }
        }
        if (!live_run(R, r, ctl)) ctl->prune = 1;  // its tiles leave the work list at this step's rebuild
    }
}

// Before a step of the device loop, for each run: the loop test and the step's settings
// (wadi2d/solver/stepper.py:106-111). The threads of one CTA; ctl->any gathers the runs' flags.
__device__ void step_settings(const StepArgs& A) {
    Ctl* ctl = A.ctl;
    const RunTab& R = A.R;
    __shared__ uint32_t any;
    if (threadIdx.x == 0) any = 0u;
    __syncthreads();
    uint32_t mine = 0u;
    for (int r = threadIdx.x; r < A.nruns; r += blockDim.x) {
        if (!live_run(R, r, ctl)) {
            R.flags[r] = 0;
            continue;
        }
        const int refresh = R.refresh_due[r] || (R.nsteps[r] % ctl->dt_every == 0);
        R.refresh_due[r] = 0;
        const int activate = (int)(R.nsteps[r] % ctl->active_every == 0);
        double dt = R.dt[r];
        const double rest = R.t_end[r] - R.t[r];
        if (rest < dt) dt = rest;
        if (ctl->dt_max < dt) dt = ctl->dt_max;
        R.dt_step[r] = dt;
        R.dtf[r] = (float)dt;
        const double t_new = R.t[r] + dt;
        R.dt_tally[r] = t_new - R.t[r];
        R.max_time[r] = (float)t_new;
        const int want_max = ctl->max_every > 0 && ((R.nsteps[r] + 1) % ctl->max_every == 0);
        const int act = activate && ctl->adaptive;
        R.flags[r] = F_RUN | (refresh ? F_WAVE : 0) | (activate ? F_WET : 0) | (want_max ? F_MAX : 0) | (act ? F_ACT : 0);
        if (refresh) R.wave_bits[r] = 0u;
        mine |= ANY_RUN | (refresh ? ANY_WAVE : 0u) | (act ? ANY_ACT : 0u) | (want_max ? ANY_MAX : 0u);
    }
    if (mine) atomicOr(&any, mine);
    __syncthreads();
    if (threadIdx.x == 0) ctl->any = any;
    // the wave of each tile of a run that refreshes: the face pass's strip form takes each half's maximum into it
    if (any & ANY_WAVE)
        for (int t = threadIdx.x; t < A.ntiles; t += blockDim.x)
            if (R.flags[A.tile_run[t]] & F_WAVE) A.wave[t] = 0.0f;
}

__global__ void prestep_kernel(StepArgs A) { step_settings(A); }

// The end of a host-driven step of run 0: the swap of the ping-pong pairs (wadi2d/solver/gpu/backend.py:185-188).
__global__ void endstep_kernel(StepArgs A) { A.R.parity[0] ^= 1; }

// A host-driven step of run 0 (the reference backend's step(dt, want_wave, want_wet)).
__global__ void setstep_kernel(StepArgs A, float dtf, int want_wave, int want_wet, int nact) {
    Ctl* ctl = A.ctl;
    ctl->nact = nact;
    ctl->nwork = nact;
    ctl->any = ANY_RUN | (want_wave ? ANY_WAVE : 0u);
    A.R.dtf[0] = dtf;
    A.R.flags[0] = F_RUN | (want_wave ? F_WAVE : 0) | (want_wet ? F_WET : 0);
    if (want_wave) A.R.wave_bits[0] = 0u;
}

// ------------------------------------------------------------------ active-list rebuild (one CTA of 1024)

// Exclusive scan of flags over one 1024-thread CTA; returns this thread's offset and the total in *total.
__device__ __forceinline__ int block_scan(int flag, int* warp_sums, int* total) {
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    int v = flag;
    for (int o = 1; o < 32; o <<= 1) {
        const int n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += n;
    }
    if (lane == 31) warp_sums[wid] = v;
    __syncthreads();
    if (wid == 0) {
        int w = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int n = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += n;
        }
        warp_sums[lane] = w;  // inclusive sums of warps
    }
    __syncthreads();
    const int before = (wid > 0 ? warp_sums[wid - 1] : 0) + v - flag;
    *total = warp_sums[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before;
}

// rebuild_active(check=True), wadi2d/solver/stepper.py:56-92, for the runs that rebuild at this step: wet or kept
// tiles and their eight neighbours are active; a tile sleeps after SLEEP_CHECKS checks in a row that did not want it;
// tiles that join the list are listed in woken for their wet share to be written. Then the work list: the active tiles
// of the runs that take another step, rebuilt whenever the active list or the set of stepping runs changed.
// only_work = 1: the work list alone, before the first step of the device loop.
__device__ void rebuild_lists(const StepArgs& A, int only_work) {
    Ctl* ctl = A.ctl;
    const bool rebuild = !only_work && (ctl->any & ANY_ACT);
    if (!only_work && !rebuild) {
        // no tile woke at this step: the plan pass that follows has nothing to do
        if (threadIdx.x == 0) ctl->nwoken = 0;
        if (!ctl->prune) return;
    }
    const int nt = A.ntiles;
    int* wet_eff = A.scratch;
    int* flags = A.scratch + nt;
    __shared__ int sums[32];
    if (rebuild) {
        for (int t = threadIdx.x; t < nt; t += blockDim.x) wet_eff[t] = t != 0 && (A.wet[t] != 0 || A.keep[t] != 0);
        __syncthreads();
        for (int t = threadIdx.x; t < nt; t += blockDim.x) {
            if (t == 0) {
                flags[0] = 0;
                continue;
            }
            const int cur = A.is_act[t];
            if (!(A.R.flags[A.tile_run[t]] & F_ACT)) {  // this tile's run does not rebuild at this step
                flags[t] = cur;
                continue;
            }
            int act = wet_eff[t];
            for (int n = 0; n < 8; ++n) act |= wet_eff[A.nbr[8 * t + n]];
            if (act)
                A.idle[t] = 0;
            else
                A.idle[t] += 1;
            act |= cur && A.idle[t] < SLEEP_CHECKS;
            flags[t] = act | ((act && !cur) << 1);
            A.is_act[t] = act;
        }
        __syncthreads();
        int nact = 0, nwoken = 0;
        for (int base = 0; base < nt; base += blockDim.x) {
            const int t = base + threadIdx.x;
            const int f = t < nt ? flags[t] : 0;
            int tot_a, tot_w;
            const int oa = block_scan(f & 1, sums, &tot_a);
            const int ow = block_scan((f >> 1) & 1, sums, &tot_w);
            if (f & 1) A.active[nact + oa] = t;
            if (f & 2) A.woken[nwoken + ow] = t;
            nact += tot_a;
            nwoken += tot_w;
        }
        if (threadIdx.x == 0) {
            ctl->nact = nact;
            ctl->nwoken = nwoken;
        }
    }
    // the work list, in tile order: active tiles whose run takes another step
    int nwork = 0;
    for (int base = 0; base < nt; base += blockDim.x) {
        const int t = base + threadIdx.x;
        const int f = t > 0 && t < nt && A.is_act[t] && live_run(A.R, A.tile_run[t], ctl);
        int tot;
        const int o = block_scan(f, sums, &tot);
        if (f) A.work[nwork + o] = t;
        nwork += tot;
    }
    if (threadIdx.x == 0) {
        ctl->nwork = nwork;
        ctl->prune = 0;
    }
}

__global__ void __launch_bounds__(1024) activity_kernel(StepArgs A, int only_work) { rebuild_lists(A, only_work); }

// The end of a step of the device loop and the settings of the next, in one CTA of 1024 threads: each running run's
// clock, the active-list rebuild (for the runs that check at this step) with the woken tiles and the work list, then
// the next step's loop test and settings. plan_kernel, after it, takes the woken tiles.
__global__ void __launch_bounds__(1024) control_kernel(StepArgs A) {
    run_clocks(A);
    __syncthreads();
    rebuild_lists(A, 0);
    __syncthreads();
    step_settings(A);
}

// refresh_plan of the listed tiles (wadi2d/solver/gpu/kernels/cells.cu:66-78) from the current mean depth. count < 0:
// the tiles the device loop's last rebuild woke (ctl->nwoken, 0 when it did not rebuild).
__global__ void __launch_bounds__(256) plan_kernel(StepArgs A, const int32_t* list, int count) {
    Ctl* ctl = A.ctl;
    if (count < 0) count = ctl->nwoken;
    for (int a = blockIdx.x; a < count; a += gridDim.x) {
        const int t = list[a];
        const int tj = A.tiles[2 * t], ti = A.tiles[2 * t + 1];
        const int base = (tj * TILE + GY) * A.px + ti * TILE + GX;
        const int ts = table_of(A, t);
        const float2* pairs_t = A.dtab2 + (size_t)ts * (A.rows - 1) * TILE2;
        const float* h = A.hh[A.R.parity[A.tile_run[t]]];
        for (int c = 0; c < 4; ++c) {
            const int jj = threadIdx.y * 4 + c, ii = threadIdx.x;
            const int local = jj * TILE + ii;
            const int k = base + jj * A.px + ii;
            A.om[k] = cell_plan(h[k], A.hc[ts * TILE2 + local], pairs_t + local, A.rows);
        }
    }
}

// Maxima.update over the active tiles, host-driven (wadi2d/engine/maxima.py:118-130): the current halves are the
// state after the step.
__global__ void __launch_bounds__(256) maxima_kernel(StepArgs A, float time, float arrive, float deep, int nact) {
    for (int a = blockIdx.x; a < nact; a += gridDim.x) {
        const int t = A.active[a];
        const int tj = A.tiles[2 * t], ti = A.tiles[2 * t + 1];
        const int base = (tj * TILE + GY) * A.px + ti * TILE + GX;
        for (int c = 0; c < 4; ++c) {
            const int jj = threadIdx.y * 4 + c, ii = threadIdx.x;
            const int k = base + jj * A.px + ii;
            const int pc = A.R.parity[A.tile_run[t]];
            envelope_cell(A, t * TILE2 + jj * TILE + ii, k, A.d[k], A.hh[pc][k], time, arrive, deep, A.uu[0][pc], A.uu[1][pc]);
        }
    }
}

// Tally.add, host-driven (wadi2d/engine/maxima.py:53-62).
__global__ void tally_kernel(StepArgs A, double dt) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= A.ntally) return;
    const float qv = A.taxis[m] ? A.q[1][A.tface[m]] : A.q[0][A.tface[m]];
    A.ttotal[m] += dt * (double)(A.tsign[m] * qv);
}

// ------------------------------------------------------------------ layout converters

// REF_TILE -> NATIVE, own cells of every allocated tile (halo entries of the reference layout are copies).
__global__ void ref_to_native_kernel(const float* __restrict__ ref, float* __restrict__ nat,
                                     const int32_t* __restrict__ tiles, int ntiles, int px) {
    const int t = blockIdx.x + 1;
    if (t >= ntiles) return;
    const int tj = tiles[2 * t], ti = tiles[2 * t + 1];
    for (int idx = threadIdx.x; idx < TILE2; idx += blockDim.x) {
        const int jj = idx / TILE, ii = idx % TILE;
        nat[(size_t)(tj * TILE + jj + GY) * px + ti * TILE + ii + GX] = ref[(size_t)t * 1296 + (jj + 2) * 36 + ii + 2];
    }
}

// NATIVE -> REF_TILE, every entry of every allocated tile: halos read the neighbour cell they copy (zero beyond
// the grid or on a missing tile, as the reference's void tile), tile 0 is zero.
__global__ void native_to_ref_kernel(const float* __restrict__ nat, float* __restrict__ ref,
                                     const int32_t* __restrict__ tiles, const int32_t* __restrict__ tile_of,
                                     int ntiles, int ny, int nx, int px) {
    const int t = blockIdx.x;
    if (t >= ntiles) return;
    for (int idx = threadIdx.x; idx < 1296; idx += blockDim.x) {
        float v = 0.0f;
        if (t > 0) {
            const int j = tiles[2 * t] * TILE + idx / 36 - 2;
            const int i = tiles[2 * t + 1] * TILE + idx % 36 - 2;
            if (j >= 0 && j < ny && i >= 0 && i < nx && tile_of[(j / TILE) * (nx / TILE) + i / TILE] != 0)
                v = nat[(size_t)(j + GY) * px + i + GX];
        }
        ref[(size_t)t * 1296 + idx] = v;
    }
}

// Tables (ntiles,32,32,rows) and (ntiles,32,32,rows,2) -> level-major pairs and quads (ntiles,rows-1,32,32).
__global__ void pack_tables_kernel(const float* __restrict__ dtab, const float* __restrict__ ftabx,
                                   const float* __restrict__ ftaby, float2* __restrict__ dtab2,
                                   float4* __restrict__ fx, float4* __restrict__ fy, int ntiles, int rows) {
    const size_t n = (size_t)ntiles * (rows - 1) * TILE2;
    for (size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
        const size_t local = o % TILE2;
        const size_t r = (o / TILE2) % (rows - 1);
        const size_t t = o / ((size_t)TILE2 * (rows - 1));
        const size_t cell = t * TILE2 + local;
        dtab2[o] = make_float2(dtab[cell * rows + r], dtab[cell * rows + r + 1]);
        const float* a = ftabx + cell * rows * 2 + 2 * r;
        fx[o] = make_float4(a[0], a[1], a[2], a[3]);
        const float* b = ftaby + cell * rows * 2 + 2 * r;
        fy[o] = make_float4(b[0], b[1], b[2], b[3]);
    }
}

// Boundary marks: clear, then one bit per boundary cell.
__global__ void bmark_kernel(StepArgs A, int clear_words) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t* mark = const_cast<uint32_t*>(A.bmark);
    if (clear_words > 0) {
        for (int w = tid; w < clear_words; w += gridDim.x * blockDim.x) mark[w] = 0u;
        return;
    }
    for (int m = tid; m < A.nb; m += gridDim.x * blockDim.x) {
        const int fid = fid_of_native(A, A.bcell[m]);
        atomicOr(mark + fid / TILE, 1u << (fid % TILE));
    }
}

#endif  // W2B_FAST

}  // namespace w2b
