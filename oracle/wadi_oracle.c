/*
 * oracle/wadi_oracle.c -- CPU restatement of Wadi2D's uniform-grid shallow-water step and of its sub-grid table
 * builder. TEST INFRASTRUCTURE ONLY: tests/, the smoke check and the benchmark's CPU-baseline leg load it as the
 * checker; the product (wadi2d_b200) never links, imports or calls it.
 *
 * Arithmetic follows the reference statement by statement so that, compiled without FMA contraction
 * (-ffp-contract=off) and without fast math, every float32 result equals the reference's Numba CPU twin bit for bit
 * (pinned by tests/test_oracle_golden.py against vectors made by running the reference itself):
 *   step kernels      wadi2d/solver/cpu/kernels.py:19-334 (= gpu/kernels/faces.cu:10-175, cells.cu:4-111)
 *   envelope / tally  wadi2d/engine/maxima.py:75-100
 *   table kernels     wadi2d/tables/core.py:16-371
 * Layout is the reference's tile-with-halo state layout (wadi2d/solver/layout.py:19-50): tile t, row j, column i,
 * k = t*STRIDE2 + j*STRIDE + i with a 2-cell halo; static tables are (ntiles, TILE, TILE, ...).
 *
 * Numba's float32 cbrt is float(cbrt(double(x))) (numba/np/npyfuncs.py np_real_cbrt_impl calls libm cbrt through
 * np.power(x, 1/3) under fastmath); cbrt32 below does the same.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define TILE 32
#define HALO 2
#define STRIDE (TILE + 2 * HALO)
#define STRIDE2 (STRIDE * STRIDE)
#define TILE2 (TILE * TILE)

/* The step section's arithmetic type: float (the reference's arithmetic, bit for bit) or, compiled with
 * -DOR_REAL_DOUBLE, double (the FP64 run that the float results are measured against; same statements, constants
 * and table values, every operation in double). */
#ifdef OR_REAL_DOUBLE
typedef double real;
#define R(x) x
#define RSQRT sqrt
#define RABS fabs
#else
typedef float real;
#define R(x) x##f
#define RSQRT sqrtf
#define RABS fabsf
#endif

typedef struct {
    real g, dx, e_wet, h_cfl, u_max, lead, a_min;
    int32_t rows, second, sheet, mirror, carry;
} OrParams;

typedef struct {
    real *h, *d, *u, *v, *mx, *my, *qx, *qy;
    real *u1, *v1, *mx1, *my1, *qx1, *qy1, *r, *src, *res, *om;
    const real *zcx, *zcy;
    const real *Hc, *dtab;
    const real *flx, *frx, *glx, *grx, *efx, *cwx, *ftabx;
    const real *fly, *fry, *gly, *gry, *efy, *cwy, *ftaby;
    real *wave;
    int32_t *wet;
} OrArrays;

int or_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

/* ------------------------------------------------------------------ float32 helpers (cpu/kernels.py:19-83) */

static inline real cbrt32(real x) { return (real)cbrt((double)x); }
static inline real fmax32(real a, real b) { return a >= b ? a : b; } /* Python max(a, b) on ordered values */
static inline real fmin32(real a, real b) { return a <= b ? a : b; }

static inline real minmod(real a, real b) {
    if (a * b <= R(0.0)) return R(0.0);
    return RABS(a) < RABS(b) ? a : b;
}

static inline real ustar(real uc, real uup, real udown, int second) {
    if (!second) return uc;
    return uc + R(0.5) * minmod(uc - uup, udown - uc);
}

static inline real gated(real neighbour, real own, int mirror) {
    return (mirror && neighbour == R(0.0)) ? own : neighbour;
}

/* cell_level, cpu/kernels.py:39-48 */
static inline real cell_level(real hb, real hc, const real *tab, int rows) {
    if (hc <= R(0.0)) return hb;
    int last = rows - 1;
    if (hb >= hc) return tab[last] + (hb - hc);
    real s = RSQRT(hb / hc) * (real)last;
    int r = (int)s;
    if (r > last - 1) r = last - 1;
    return tab[r] + (s - (real)r) * (tab[r + 1] - tab[r]);
}

/* cell_plan, cpu/kernels.py:51-59 */
static inline real cell_plan(real hb, real hc, const real *tab, int rows) {
    if (hc <= R(0.0) || hb >= hc) return R(1.0);
    int last = rows - 1;
    real s = RSQRT(hb / hc) * (real)last;
    int r = (int)s;
    if (r > last - 1) r = last - 1;
    real m = (real)last;
    return hc * (real)(2 * r + 1) / (m * m) / fmax32(tab[r + 1] - tab[r], R(1e-12));
}

/* face_lookup, cpu/kernels.py:62-83 */
static inline void face_lookup(real e, real top, const real *tab, int rows, real *A, real *T, real *W) {
    int last = rows - 1;
    real m = (real)last;
    if (e >= top) {
        real a1 = tab[2 * last];
        real a0 = tab[2 * last - 2];
        real c = (m - R(1.0)) / m;
        real w = (a1 - a0) / (top * (R(1.0) - c * c));
        real area = a1 + w * (e - top);
        *A = area;
        *T = tab[2 * last + 1] * (area / fmax32(a1, R(1e-12)));
        *W = w;
        return;
    }
    real s = RSQRT(e / top) * m;
    int r = (int)s;
    if (r > last - 1) r = last - 1;
    real c0 = (real)r / m;
    real c1 = (real)(r + 1) / m;
    real e0 = c0 * c0 * top;
    real de = (c1 * c1 - c0 * c0) * top;
    real f = (e - e0) / de;
    real a0 = tab[2 * r];
    real a1 = tab[2 * r + 2];
    real t0 = tab[2 * r + 1];
    *A = a0 + f * (a1 - a0);
    *T = t0 + f * (tab[2 * r + 3] - t0);
    *W = (a1 - a0) / de;
}

/* face_step, cpu/kernels.py:86-219. s: array step along the face normal, p: across it. Returns the wave speed. */
static real face_step(int k, int fid, real dt, int want_wave, const OrParams *P, const real *om, const real *zc,
                       int s, int p, const real *h, const real *d, const real *u, const real *m, const real *q,
                       const real *qp, const real *vp, const real *fl, const real *fr, const real *gl,
                       const real *gr, const real *ef, const real *cw, const real *ftab, real *u1, real *m1,
                       real *q1) {
    const real ZERO = R(0.0), HALF = R(0.5), ONE = R(1.0);
    const int rows = P->rows;
    const real dx = P->dx;
    const real span = dx;
    real e_l = d[k - s] - fl[fid];
    real e_r = d[k] - fr[fid];
    real uf = u[k];
    real e_lp = fmax32(e_l, ZERO);
    real e_rp = fmax32(e_r, ZERO);
    int from_left = uf > ZERO || (uf == ZERO && e_l >= e_r);
    real eup = from_left ? e_lp : e_rp;
    if (eup <= P->e_wet) {
        u1[k] = ZERO;
        m1[k] = ZERO;
        q1[k] = ZERO;
        return ZERO;
    }
    real eface = eup;
    if (P->carry && cw[fid] == ZERO) {
        real dz = from_left ? (zc[k - s] - fl[fid]) : (zc[k] - fr[fid]);
        if (dz > R(1e-6)) {
            real phi = (eup - R(2.0) * dz) / (R(2.0) * dz);
            phi = phi < ZERO ? ZERO : (phi > ONE ? ONE : phi);
            eface = eup - phi * dz;
        }
    }
    const real *tab = ftab + (size_t)2 * rows * fid;
    real area, t, w;
    face_lookup(eface, ef[fid], tab, rows, &area, &t, &w);
    real h_l = h[k - s];
    real h_r = h[k];
    real hup = from_left ? h_l : h_r;

    /* [1] section */
    real rho = ONE;
    real d_eta = e_rp - e_lp;
    if (P->sheet) {
        real avol = hup * dx;
        real edown = from_left ? e_rp : e_lp;
        if (avol < area) {
            real sub = fmin32(e_lp, e_rp) / fmax32(e_lp, e_rp);
            real sub2 = sub * sub;
            real alpha = sub2 * sub2;
            rho = alpha + (ONE - alpha) * avol / area;
        }
        if (edown <= ZERO) {
            /* [2] disconnected */
            real g_u = from_left ? gl[fid] : gr[fid];
            real g_d = from_left ? gr[fid] : gl[fid];
            real h_d = from_left ? h_r : h_l;
            real drop = (hup - g_u) - fmax32(h_d - g_d, HALF * (g_u - g_d));
            real level_drop = RABS(e_l - e_r);
            real drive = fmax32(eup, fmin32(drop, level_drop));
            d_eta = from_left ? -drive : drive;
        }
    }

    /* [3] momentum fluxes */
    const int mirror = P->mirror, second = P->second;
    real um = gated(u[k - s], uf, mirror);
    real up = gated(u[k + s], uf, mirror);
    real umm = gated(u[k - 2 * s], um, mirror);
    real upp = gated(u[k + 2 * s], up, mirror);
    real qc_l = HALF * (q[k - s] + q[k]);
    real qc_r = HALF * (q[k] + q[k + s]);
    real s_l = qc_l > ZERO ? ustar(um, umm, uf, second) : ustar(uf, up, um, second);
    real s_r = qc_r > ZERO ? ustar(uf, um, up, second) : ustar(up, upp, uf, second);
    real flux = qc_r * s_r - qc_l * s_l;
    real qy_s = HALF * (qp[k - s] + qp[k]);
    real qy_n = HALF * (qp[k - s + p] + qp[k + p]);
    real u_s = gated(u[k - p], uf, mirror);
    real u_n = gated(u[k + p], uf, mirror);
    real uss = gated(u[k - 2 * p], u_s, mirror);
    real unn = gated(u[k + 2 * p], u_n, mirror);
    real us_s = qy_s > ZERO ? ustar(u_s, uss, uf, second) : ustar(uf, u_n, u_s, second);
    real us_n = qy_n > ZERO ? ustar(uf, u_s, u_n, second) : ustar(u_n, unn, uf, second);
    flux += qy_n * us_n - qy_s * us_s;

    /* [4] momentum and pressure */
    real abar = HALF * (h_l + h_r) * dx;
    real press = dt * P->g * d_eta / span;
    real us;
    if (abar > R(1e-6) * dx)
        us = (m[k] - dt * flux / span) / abar - press;
    else
        us = uf - press;

    /* [5] friction */
    real vb = R(0.25) * (vp[k - s] + vp[k] + vp[k - s + p] + vp[k + p]);
    real t3 = t * t * t * cbrt32(t);
    real fric = area * area / fmax32(t3, R(1e-30));
    if (rho < ONE) fric = fric / fmax32(rho * cbrt32(rho), R(1e-12));
    real a = dt * P->g * fric;
    real sp = RSQRT(us * us + vb * vb);
    real un = R(2.0) * us / (ONE + RSQRT(ONE + R(4.0) * a * sp));
    if (RABS(un) > P->u_max) un = un > ZERO ? P->u_max : -P->u_max;

    /* [6] crest face */
    real qn = area * rho * un;
    real c = cw[fid];
    if (c != ZERO) {
        real area_c = area, w_c = w;
        if (c < ZERO) {
            c = -c;
            real ua = from_left ? um : up;
            real tc;
            face_lookup(eup + HALF * ua * ua / P->g, ef[fid], tab, rows, &area_c, &tc, &w_c);
        }
        real qc = c * area_c * RSQRT(area_c / fmax32(w_c, R(1e-9)));
        if (RABS(qn) > qc) {
            qn = qn > ZERO ? qc : -qc;
            un = qn / fmax32(area * rho, R(1e-12));
        }
    }
    u1[k] = un;
    m1[k] = abar * un;
    q1[k] = qn;
    if (!want_wave) return ZERO;
    if (!isfinite(un)) return R(1e30);
    real d_left = d[k - s];
    real d_right = d[k];
    real dup = from_left ? d_left : d_right;
    if (dup <= P->h_cfl) return ZERO;
    real plan = from_left ? om[k - s] : om[k];
    real dother = from_left ? d_right : d_left;
    if (dother > P->h_cfl) plan = fmin32(plan, from_left ? om[k] : om[k - s]);
    real wave = RSQRT(fmax32(P->g * area * rho / (fmax32(plan, P->a_min) * dx), ZERO));
    return RABS(un) + fmin32(P->lead * RABS(un - uf), R(2.0) * wave) + wave;
}

/* faces, cpu/kernels.py:222-244 */
void or_faces(const OrArrays *A, const OrParams *P, const int32_t *active, int nact, real dt, int want_wave) {
#pragma omp parallel for schedule(dynamic, 4)
    for (int a = 0; a < nact; ++a) {
        int t = active[a];
        real w = R(0.0);
        for (int j = 0; j < TILE; ++j) {
            for (int i = 0; i < TILE; ++i) {
                int k = t * STRIDE2 + (j + HALO) * STRIDE + i + HALO;
                int fid = t * TILE2 + j * TILE + i;
                real wx = face_step(k, fid, dt, want_wave, P, A->om, A->zcx, 1, STRIDE, A->h, A->d, A->u, A->mx, A->qx,
                                     A->qy, A->v, A->flx, A->frx, A->glx, A->grx, A->efx, A->cwx, A->ftabx, A->u1, A->mx1,
                                     A->qx1);
                real wy = face_step(k, fid, dt, want_wave, P, A->om, A->zcy, STRIDE, 1, A->h, A->d, A->v, A->my, A->qy,
                                     A->qx, A->u, A->fly, A->fry, A->gly, A->gry, A->efy, A->cwy, A->ftaby, A->v1, A->my1,
                                     A->qy1);
                w = fmax32(w, fmax32(wx, wy));
            }
        }
        if (want_wave) A->wave[t] = w;
    }
}

/* limit, cpu/kernels.py:247-262 */
void or_limit(const OrArrays *A, const OrParams *P, const int32_t *active, int nact, real dt) {
    const real dx = P->dx;
    const real area = dx * dx;
#pragma omp parallel for schedule(static)
    for (int a = 0; a < nact; ++a) {
        int t = active[a];
        for (int j = 0; j < TILE; ++j) {
            for (int i = 0; i < TILE; ++i) {
                int k = t * STRIDE2 + (j + HALO) * STRIDE + i + HALO;
                real out = fmax32(A->qx1[k + 1], R(0.0)) + fmax32(-A->qx1[k], R(0.0)) + fmax32(A->qy1[k + STRIDE], R(0.0)) +
                            fmax32(-A->qy1[k], R(0.0));
                real have = fmax32(A->h[k], R(0.0)) * area;
                A->r[k] = out * dt > have ? have / (out * dt) : R(1.0);
            }
        }
    }
}

static inline real scaled(real q, real rl, real rr) { return q * (q > R(0.0) ? rl : rr); }

/* update, cpu/kernels.py:270-299 (debt = False on the uniform step) */
void or_update(const OrArrays *A, const OrParams *P, const int32_t *active, int nact, real dt, int want_plan) {
    const int rows = P->rows;
    const real dx = P->dx;
    const real area = dx * dx;
#pragma omp parallel for schedule(static)
    for (int a = 0; a < nact; ++a) {
        int t = active[a];
        int any_wet = 0;
        for (int j = 0; j < TILE; ++j) {
            for (int i = 0; i < TILE; ++i) {
                int k = t * STRIDE2 + (j + HALO) * STRIDE + i + HALO;
                int fid = t * TILE2 + j * TILE + i;
                const real *r = A->r;
                real rc = r[k];
                real qw = scaled(A->qx1[k], r[k - 1], rc);
                real qe = scaled(A->qx1[k + 1], rc, r[k + 1]);
                real qn = scaled(A->qy1[k], r[k - STRIDE], rc);
                real qs = scaled(A->qy1[k + STRIDE], rc, r[k + STRIDE]);
                A->qx[k] = qw;
                A->qy[k] = qn;
                real h0 = A->h[k];
                real inc = A->res[k] + dt * A->src[k] - dt * (qe - qw + qs - qn) / area;
                real total = h0 + inc;
                real hn = fmax32(total, R(0.0));
                A->res[k] = total > R(0.0) ? inc - (total - h0) : R(0.0);
                A->h[k] = hn;
                const real *tab = A->dtab + (size_t)rows * fid;
                A->d[k] = cell_level(hn, A->Hc[fid], tab, rows);
                if (want_plan) A->om[k] = cell_plan(hn, A->Hc[fid], tab, rows);
                if (hn > R(0.0)) any_wet = 1;
            }
        }
        A->wet[t] = any_wet;
    }
}

/* plan, cpu/kernels.py:302-311 */
void or_plan(const OrArrays *A, const OrParams *P, const int32_t *tiles, int n) {
    const int rows = P->rows;
#pragma omp parallel for schedule(static)
    for (int a = 0; a < n; ++a) {
        int t = tiles[a];
        for (int j = 0; j < TILE; ++j)
            for (int i = 0; i < TILE; ++i) {
                int k = t * STRIDE2 + (j + HALO) * STRIDE + i + HALO;
                int fid = t * TILE2 + j * TILE + i;
                A->om[k] = cell_plan(A->h[k], A->Hc[fid], A->dtab + (size_t)rows * fid, rows);
            }
    }
}

/* exchange, cpu/kernels.py:314-319 */
void or_exchange(const int32_t *active, int nact, const int32_t *slot, const int32_t *src, int nhalo, real *a) {
#pragma omp parallel for schedule(static)
    for (int n = 0; n < nact; ++n) {
        int t = active[n];
        for (int m = 0; m < nhalo; ++m) a[t * STRIDE2 + slot[m]] = a[src[(size_t)(t - 1) * nhalo + m]];
    }
}

/* boundary, cpu/kernels.py:322-334 (sequential: a follow cell reads its reference after earlier ones are set) */
void or_boundary(int n, const int32_t *cell, const int32_t *ref, const int32_t *kind, const real *d0, const real *h0,
                 real *h, real *d) {
    for (int m = 0; m < n; ++m) {
        int k = cell[m];
        if (kind[m] == 0) {
            h[k] = h0[m];
            d[k] = d0[m];
        } else if (kind[m] == 1) {
            h[k] = R(0.0);
            d[k] = R(0.0);
        } else {
            h[k] = h[ref[m]];
            d[k] = fmax32(d[ref[m]] + d0[m], R(0.0));
        }
    }
}

/* maxima, engine/maxima.py:75-92. The literal 0.5 is a float64, so the centre speed is formed in float64 and each
 * envelope entry takes the float32 rounding of its new maximum. */
void or_maxima(const int32_t *active, int nact, real time, real arrive, real deep, const real *d, const real *h,
               const real *u, const real *v, real *dmax, real *hmax, real *smax, real *zmax, real *tarr) {
#pragma omp parallel for schedule(static)
    for (int a = 0; a < nact; ++a) {
        int t = active[a];
        for (int j = 0; j < TILE; ++j)
            for (int i = 0; i < TILE; ++i) {
                int k = t * STRIDE2 + (j + HALO) * STRIDE + i + HALO;
                real dk = d[k];
                dmax[k] = fmax32(dmax[k], dk);
                hmax[k] = fmax32(hmax[k], h[k]);
                if (dk > deep) {
                    double uc = 0.5 * (double)(u[k] + u[k + 1]);
                    double vc = 0.5 * (double)(v[k] + v[k + STRIDE]);
                    double s = sqrt(uc * uc + vc * vc);
                    double sm = (double)smax[k];
                    smax[k] = (real)(sm >= s ? sm : s);
                    double hz = s * (double)dk;
                    double zm = (double)zmax[k];
                    zmax[k] = (real)(zm >= hz ? zm : hz);
                }
                if (tarr[k] < R(0.0) && dk >= arrive) tarr[k] = time;
            }
    }
}

/* tally, engine/maxima.py:95-100 and :171-182 (the device form: one FP64 total per face, dt * sign * q) */
void or_tally(int n, double dt, const int32_t *face, const int32_t *axis, const real *sign, const real *qx,
              const real *qy, double *total) {
    for (int m = 0; m < n; ++m) {
        real q = axis[m] ? qy[face[m]] : qx[face[m]];
        total[m] += dt * (double)(sign[m] * q);
    }
}

/* ------------------------------------------------------------------ table builder (tables/core.py), float64 */

static int cmp_double(const void *a, const void *b) {
    double x = *(const double *)a, y = *(const double *)b;
    return (x > y) - (x < y);
}

/* _cell_table, tables/core.py:16-41. z: n pixels (any order); tab: rows values. out3 = (zmin, relmean, hc). */
void or_cell_table(const double *z, int n, int rows, double *tab, double *out3, double *work) {
    double *p = work;        /* n */
    double *hbar_at = work + n; /* n */
    memcpy(p, z, sizeof(double) * (size_t)n);
    qsort(p, (size_t)n, sizeof(double), cmp_double);
    double zmin = p[0];
    for (int q = 0; q < n; ++q) p[q] = p[q] - zmin; /* rel */
    double c = 0.0;
    for (int q = 0; q < n; ++q) c += p[q];
    double relmean = c / (double)n;
    double hc = p[n - 1] - relmean;
    out3[0] = zmin;
    out3[1] = relmean;
    if (hc <= 1e-9) {
        for (int r = 0; r < rows; ++r) tab[r] = 0.0;
        out3[2] = 0.0;
        return;
    }
    double cum = 0.0;
    for (int m = 0; m < n; ++m) {
        cum += p[m];
        hbar_at[m] = (p[m] * (double)(m + 1) - cum) / (double)n;
    }
    int last = rows - 1;
    int m = 0;
    for (int r = 0; r < rows; ++r) {
        double x = (double)r / (double)last;
        double hb = hc * (x * x);
        while (m + 1 < n && hbar_at[m + 1] <= hb) m += 1;
        tab[r] = p[m] + (hb - hbar_at[m]) * (double)n / (double)(m + 1);
    }
    tab[last] = p[n - 1];
    out3[2] = hc;
}

/* _face_table, tables/core.py:44-79. prof is modified (raised to the crest). Returns via out2 = (zf, top). */
void or_face_table(double *prof, int m, double crest, double pixel, double n_inv, const double *weight, double length,
                   double e_lo, double e_hi, int rows, double *tab, double *out2) {
    if (!isnan(crest))
        for (int q = 0; q < m; ++q) prof[q] = prof[q] >= crest ? prof[q] : crest; /* np.maximum */
    double zf = prof[0];
    for (int q = 1; q < m; ++q)
        if (prof[q] < zf) zf = prof[q];
    double relmax = prof[0] - zf;
    for (int q = 1; q < m; ++q)
        if (prof[q] - zf > relmax) relmax = prof[q] - zf;
    double lo = relmax <= e_hi ? relmax : e_hi;
    double top = lo >= e_lo ? lo : e_lo;
    int last = rows - 1;
    for (int r = 0; r < rows; ++r) {
        double x = (double)r / (double)last;
        double e = top * (x * x);
        double area = 0.0, conv = 0.0;
        for (int q = 0; q < m; ++q) {
            double dep = e - (prof[q] - zf);
            if (dep > 0.0) {
                area += dep;
                double cb = cbrt(dep);
                conv += weight[q] * dep * (cb * cb);
            }
        }
        tab[2 * r] = pixel * area * length;
        tab[2 * r + 1] = pow(pixel * n_inv * conv * length, 0.6);
    }
    out2[0] = zf;
    out2[1] = top;
}

/* _local_radius_conveyance, tables/core.py:82-179. work: 6*(n+1) doubles + 2*n int64. */
void or_local_radius(const double *ext, int n, int i0, int i1, double zf, double top, double pixel, double n_inv,
                     const double *weight, double length, double beta, int rows, double *tab, double *work,
                     int64_t *iwork) {
    double *d = work, *per = work + n, *s0 = work + 2 * n, *s1 = s0 + (n + 1), *p0 = s1 + (n + 1),
           *p1 = p0 + (n + 1);
    int64_t *run_lo = iwork, *run_hi = iwork + n;
    for (int t = 0; t < n; ++t) run_lo[t] = run_hi[t] = 0;
    s0[0] = s1[0] = p0[0] = p1[0] = 0.0;
    double pix2 = pixel * pixel;
    int last = rows - 1;
    for (int r = 0; r < rows; ++r) {
        double x = (double)r / (double)last;
        double level = zf + top * (x * x);
        for (int t = 0; t < n; ++t) {
            double dep = level - ext[t];
            d[t] = dep > 0.0 ? dep : 0.0;
        }
        for (int t = 0; t < n; ++t) per[t] = 0.0;
        if (d[0] > 0.0) per[0] += 0.5 * pixel;
        if (d[n - 1] > 0.0) per[n - 1] += 0.5 * pixel;
        for (int t = 0; t < n - 1; ++t) {
            int wa = d[t] > 0.0, wb = d[t + 1] > 0.0;
            if (!(wa || wb)) continue;
            double rise = ext[t + 1] - ext[t];
            double seg = sqrt(pix2 + rise * rise);
            if (wa && wb) {
                per[t] += 0.5 * seg;
                per[t + 1] += 0.5 * seg;
            } else if (wa) {
                if (rise > 0.0) {
                    double f = d[t] / rise;
                    per[t] += (f <= 1.0 ? f : 1.0) * seg;
                } else {
                    per[t] += 0.5 * pixel;
                }
            } else if (-rise > 0.0) {
                double f = d[t + 1] / -rise;
                per[t + 1] += (f <= 1.0 ? f : 1.0) * seg;
            } else {
                per[t + 1] += 0.5 * pixel;
            }
        }
        int64_t start = -1;
        for (int t = 0; t < n; ++t) {
            if (d[t] > 0.0) {
                if (start < 0) start = t;
                run_lo[t] = start;
            } else {
                start = -1;
            }
        }
        int64_t end = -1;
        for (int t = n - 1; t >= 0; --t) {
            if (d[t] > 0.0) {
                if (end < 0) end = t;
                run_hi[t] = end;
            } else {
                end = -1;
            }
        }
        for (int t = 0; t < n; ++t) {
            s0[t + 1] = s0[t] + d[t];
            s1[t + 1] = s1[t] + (double)t * d[t];
            p0[t + 1] = p0[t] + per[t];
            p1[t + 1] = p1[t] + (double)t * per[t];
        }
        double conv = 0.0;
        for (int i = i0; i < i1; ++i) {
            double di = d[i];
            if (di <= 0.0) continue;
            double w = beta * di / pixel;
            if (w < 1e-9) w = 1e-9;
            int64_t lo = (int64_t)ceil((double)i - w);
            if (run_lo[i] > lo) lo = run_lo[i];
            int64_t hi = (int64_t)floor((double)i + w);
            if (run_hi[i] < hi) hi = run_hi[i];
            double fi = (double)i;
            double a_sum = (1.0 - fi / w) * (s0[i + 1] - s0[lo]) + (s1[i + 1] - s1[lo]) / w;
            a_sum += (1.0 + fi / w) * (s0[hi + 1] - s0[i + 1]) - (s1[hi + 1] - s1[i + 1]) / w;
            double p_sum = (1.0 - fi / w) * (p0[i + 1] - p0[lo]) + (p1[i + 1] - p1[lo]) / w;
            p_sum += (1.0 + fi / w) * (p0[hi + 1] - p0[i + 1]) - (p1[hi + 1] - p1[i + 1]) / w;
            double radius = p_sum > 0.0 ? pixel * a_sum / p_sum : di;
            double cb = cbrt(radius);
            conv += weight[i - i0] * di * (cb * cb);
        }
        tab[2 * r + 1] = pow(pixel * n_inv * conv * length, 0.6);
    }
}

/* window_top, tables/core.py:354-362 */
static double window_top(const double *line, int n, double zf, double top, double e_hi) {
    double hi = -INFINITY;
    for (int t = 0; t < n; ++t)
        if (line[t] > hi) hi = line[t];
    double rel = hi - zf;
    double cap = rel <= e_hi ? rel : e_hi;
    return top >= cap ? top : cap;
}

static inline double lined(double pixel_n, double cell_n) { return isnan(pixel_n) ? 1.0 : cell_n / pixel_n; }

/*
 * One tile, tables/core.py:188-264 (tile_tables) followed, when local != 0, by tables/core.py:282-351
 * (tile_local_radius). zbig: (W + 2*margin) square pixel block, W = TILE*k + 1, row-major; the core block of
 * tile_tables is zbig[margin:margin+W, margin:margin+W]. npix: W x W Manning n per pixel or NULL (no lining).
 * Per-cell inputs nman, xcrest, xlen, ycrest, ylen are (TILE, TILE). Outputs (TILE, TILE[, rows[, 2]]) float64.
 */
void or_tile_tables(const double *zbig, int margin, int k, double pixel, const double *nman, const double *npix,
                    const double *xcrest, const double *xlen, const double *ycrest, const double *ylen, double e_lo,
                    double e_hi, int rows, int local, double beta, double *zmin, double *relmean, double *hc,
                    double *dtab, double *zfx, double *efx, double *ftabx, double *zfy, double *efy, double *ftaby) {
    const int W = TILE * k + 1;
    const int B = W + 2 * margin;
#define ZC(r, c) zbig[(size_t)((r) + margin) * B + (c) + margin]
#define ZB(r, c) zbig[(size_t)(r) * B + (c)]
#define NP(r, c) npix[(size_t)(r) * W + (c)]
    int lined_ = npix != NULL;
#pragma omp parallel
    {
        double *cell = malloc(sizeof(double) * (size_t)k * k);
        double *cwork = malloc(sizeof(double) * 2 * (size_t)k * k);
        double *prof = malloc(sizeof(double) * (size_t)k);
        double *weight = malloc(sizeof(double) * (size_t)k);
        int nfull = k + 2 * margin;
        double *full = malloc(sizeof(double) * (size_t)nfull);
        double *lwork = malloc(sizeof(double) * (6 * (size_t)nfull + 8));
        int64_t *liwork = malloc(sizeof(int64_t) * (2 * (size_t)nfull + 2));
        double out[3];
#pragma omp for schedule(dynamic, 1)
        for (int j = 0; j < TILE; ++j) {
            for (int i = 0; i < TILE; ++i) {
                int c = j * TILE + i;
                int r0 = 1 + j * k, c0 = 1 + i * k;
                for (int a = 0; a < k; ++a)
                    for (int b = 0; b < k; ++b) cell[a * k + b] = ZC(r0 + a, c0 + b);
                or_cell_table(cell, k * k, rows, dtab + (size_t)c * rows, out, cwork);
                zmin[c] = out[0];
                relmean[c] = out[1];
                hc[c] = out[2];
                for (int q = 0; q < k; ++q) {
                    double near = ZC(r0 + q, c0), far = ZC(r0 + q, c0 - 1);
                    prof[q] = far >= near ? far : near;
                    weight[q] = lined_ ? lined(far > near ? NP(r0 + q, c0 - 1) : NP(r0 + q, c0), nman[c]) : 1.0;
                }
                or_face_table(prof, k, xcrest[c], pixel, 1.0 / nman[c], weight, xlen[c], e_lo, e_hi, rows,
                              ftabx + (size_t)c * 2 * rows, out);
                zfx[c] = out[0];
                efx[c] = out[1];
                for (int q = 0; q < k; ++q) {
                    double near = ZC(r0, c0 + q), far = ZC(r0 - 1, c0 + q);
                    prof[q] = far >= near ? far : near;
                    weight[q] = lined_ ? lined(far > near ? NP(r0 - 1, c0 + q) : NP(r0, c0 + q), nman[c]) : 1.0;
                }
                or_face_table(prof, k, ycrest[c], pixel, 1.0 / nman[c], weight, ylen[c], e_lo, e_hi, rows,
                              ftaby + (size_t)c * 2 * rows, out);
                zfy[c] = out[0];
                efy[c] = out[1];
                if (!local) continue;
                /* tables/core.py:324-351 */
                for (int axis = 0; axis < 2; ++axis) {
                    const double *crest = axis == 0 ? xcrest : ycrest;
                    const double *len = axis == 0 ? xlen : ylen;
                    double *zf = axis == 0 ? zfx : zfy;
                    double *ef = axis == 0 ? efx : efy;
                    double *ftab = (axis == 0 ? ftabx : ftaby) + (size_t)c * 2 * rows;
                    if (!isnan(crest[c])) continue;
                    for (int t = 0; t < nfull; ++t) {
                        double x0, x1;
                        if (axis == 0) {
                            x0 = ZB(r0 + t, margin + c0 - 1);
                            x1 = ZB(r0 + t, margin + c0);
                        } else {
                            x0 = ZB(margin + r0 - 1, c0 + t);
                            x1 = ZB(margin + r0, c0 + t);
                        }
                        full[t] = x0 >= x1 ? x0 : x1;
                    }
                    for (int q = 0; q < k; ++q) {
                        if (!lined_) {
                            weight[q] = 1.0;
                            continue;
                        }
                        double near, far, pn_far, pn_near;
                        if (axis == 0) {
                            near = ZB(margin + r0 + q, margin + c0);
                            far = ZB(margin + r0 + q, margin + c0 - 1);
                            pn_far = NP(r0 + q, c0 - 1);
                            pn_near = NP(r0 + q, c0);
                        } else {
                            near = ZB(margin + r0, margin + c0 + q);
                            far = ZB(margin + r0 - 1, margin + c0 + q);
                            pn_far = NP(r0 - 1, c0 + q);
                            pn_near = NP(r0, c0 + q);
                        }
                        weight[q] = lined(far > near ? pn_far : pn_near, nman[c]);
                    }
                    /* _raise_top, tables/core.py:365-371 */
                    double top = window_top(full, nfull, zf[c], ef[c], e_hi);
                    if (top > ef[c]) {
                        for (int q = 0; q < k; ++q) prof[q] = full[margin + q];
                        or_face_table(prof, k, NAN, pixel, 1.0 / nman[c], weight, len[c], top, e_hi, rows, ftab, out);
                        zf[c] = out[0];
                        ef[c] = out[1];
                    }
                    int e = (int)ceil(beta * ef[c] / pixel);
                    if (e > margin) e = margin;
                    or_local_radius(full + (margin - e), k + 2 * e, e, e + k, zf[c], ef[c], pixel, 1.0 / nman[c],
                                    weight, len[c], beta, rows, ftab, lwork, liwork);
                }
            }
        }
        free(cell);
        free(cwork);
        free(prof);
        free(weight);
        free(full);
        free(lwork);
        free(liwork);
    }
#undef ZC
#undef ZB
#undef NP
}
