/*
 * mpm2.c -- the 2D MLS-MPM/APIC step (Flip.java) and the 2D sort by cell
 * (Scatter.java sortCount/cell/cellStarts + CountingSort), restated in C.
 *
 * Test infrastructure only (see oracle.h). Every expression keeps the operand
 * order of the IR the reference builds; comments give the file:line followed.
 * Paths are relative to vexelray-sim-fluid-core/src/main/java/dev/vexelray/sim/fluid/.
 */
#include "oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* Body.clamp, Body.min, Body.max on f32 */
static inline float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

/* particle/Flip.java:102-107: DT 0, GX 1, GY 2, BULK 3, RHO0 4 */
enum { P_DT = 0, P_GX = 1, P_GY = 2, P_BULK = 3, P_RHO0 = 4 };

/* particle/Flip.java:128-131 */
static const float WALL = 1.0f;
static const int WALL_NODE = 1;
/* particle/Flip.java:316 */
static const float EMPTY = 1e-9f;
/* particle/Flip.java:430 */
static const float J_BOUND = 10.0f;

/* The pressure's impulse factor s = 4*dt*V0*J*p (Flip.java:283-286).
 * REF: J*p = B*(1 - J). TAIT: p = k((1/J)^7 - 1), so J*p = k*(J^-6 - J). */
static inline float impulse(float dt, float m, float rho0, float bulk, float j, int eos) {
    float jp;
    if (eos == OR_EOS_TAIT) {
        float r = 1.0f / j;
        float r2 = r * r;
        float r6 = (r2 * r2) * r2;
        jp = bulk * (r6 - j);
    } else {
        jp = bulk * (1.0f - j);
    }
    return (4.0f * (dt * (m / rho0))) * jp;
}

/* Flip.Stencil.of (Flip.java:572-581) and weights (584-590). */
typedef struct { int base; float fx, fy; float wx[3], wy[3]; } stencil2;

static inline void weights(float f, float w[3]) {
    float a = 1.5f - f;
    float c = f - 1.0f;
    float e = f - 0.5f;
    w[0] = 0.5f * (a * a);
    w[1] = 0.75f - c * c;
    w[2] = 0.5f * (e * e);
}

static inline stencil2 stencil_of(float px, float py, int nx, int ny) {
    stencil2 s;
    float x = clampf(px, 0.5f, (float)nx - 1.5f);
    float y = clampf(py, 0.5f, (float)ny - 1.5f);
    int col = (int)fminf(x - 0.5f, (float)(nx - 3));
    int row = (int)fminf(y - 0.5f, (float)(ny - 3));
    s.fx = x - (float)col;
    s.fy = y - (float)row;
    s.base = row * nx + col;
    weights(s.fx, s.wx);
    weights(s.fy, s.wy);
    return s;
}

void or_flip2_clear(or_flip2* s) {                                   /* Flip.java:226-235 */
    size_t n = (size_t)s->nx * s->ny;
    memset(s->gm, 0, n * sizeof(float));
    memset(s->gmu, 0, n * sizeof(float));
    memset(s->gmv, 0, n * sizeof(float));
}

void or_flip2_scatter(or_flip2* s, const float* params, or_physics ph) {   /* Flip.java:269-303 */
    const int nx = s->nx, ny = s->ny;
    const float dt = params[P_DT], bulk = params[P_BULK], rho0 = params[P_RHO0];
    for (int p = 0; p < s->np; p++) {
        stencil2 st = stencil_of(s->x[p], s->y[p], nx, ny);
        float m = s->m[p], u = s->u[p], w = s->v[p];
        float c00 = s->c00[p], c01 = s->c01[p], c10 = s->c10[p], c11 = s->c11[p];
        float sp = impulse(dt, m, rho0, bulk, s->j[p], ph.eos);
        for (int k = 0; k < 9; k++) {
            float wgt = st.wx[k % 3] * st.wy[k / 3];                   /* Flip.java:592-594 */
            float wm = wgt * m;
            float dx = (float)(k % 3) - st.fx;                         /* Flip.java:597-603 */
            float dy = (float)(k / 3) - st.fy;
            float velU = u + (c00 * dx + c01 * dy);
            float velV = w + (c10 * dx + c11 * dy);
            int node = st.base + (k / 3) * nx + k % 3;                 /* Scatter.java:433 */
            s->gm[node] += wm;
            s->gmu[node] += wm * velU + wgt * (sp * dx);
            s->gmv[node] += wm * velV + wgt * (sp * dy);
        }
    }
}

void or_flip2_grid(or_flip2* s, const float* params, or_physics ph) {      /* Flip.java:366-412 */
    const int nx = s->nx, ny = s->ny;
    const float dt = params[P_DT], gx = params[P_GX], gy = params[P_GY];
    for (int node = 0; node < nx * ny; node++) {
        int ni = node % nx;
        int nj = node / nx;
        float m = s->gm[node];
        float u = 0.0f, w = 0.0f;
        if (m > EMPTY) {
            float weight = 1.0f;
            u = s->gmu[node] / m + dt * (gx * weight);
            w = s->gmv[node] / m + dt * (gy * weight);
        }
        if (ph.sticky > 0) {
            int t = ph.sticky;
            if (ni < t || ni > nx - 1 - t || nj < t || nj > ny - 1 - t) { u = 0.0f; w = 0.0f; }
        } else {
            if (!(ni > WALL_NODE)) u = fmaxf(u, 0.0f);
            if (ni > nx - 2 - WALL_NODE) u = fminf(u, 0.0f);
            if (!(nj > WALL_NODE)) w = fmaxf(w, 0.0f);
            if (nj > ny - 2 - WALL_NODE) w = fminf(w, 0.0f);
        }
        s->gu[node] = u;
        s->gv[node] = w;
    }
}

/* Flip.keepInside (Flip.java:548-559) */
static inline void keep_inside(float* at, float* vel, int size) {
    float lo = WALL;
    float hi = (float)size - 1.0f - WALL;
    if (*at < lo) { *at = lo; *vel = fmaxf(*vel, 0.0f); }
    if (*at > hi) { *at = hi; *vel = fminf(*vel, 0.0f); }
}

static void advect2(or_flip2* s, const float* params, int relax) {   /* Flip.java:494-545 */
    const int nx = s->nx, ny = s->ny;
    const float dt = params[P_DT];
    for (int p = 0; p < s->np; p++) {
        stencil2 st = stencil_of(s->x[p], s->y[p], nx, ny);
        float u = 0, w = 0, b00 = 0, b01 = 0, b10 = 0, b11 = 0, density = 0;
        for (int k = 0; k < 9; k++) {
            float wgt = st.wx[k % 3] * st.wy[k / 3];
            float dx = (float)(k % 3) - st.fx;
            float dy = (float)(k / 3) - st.fy;
            int node = st.base + (k / 3) * nx + k % 3;
            float ui = wgt * s->gu[node];
            float vi = wgt * s->gv[node];
            u = u + ui;
            w = w + vi;
            if (relax) density = density + wgt * s->gm[node];         /* Flip.java:512-514 */
            b00 = b00 + ui * dx;
            b01 = b01 + ui * dy;
            b10 = b10 + vi * dx;
            b11 = b11 + vi * dy;
        }
        float c00 = 4.0f * b00, c01 = 4.0f * b01, c10 = 4.0f * b10, c11 = 4.0f * b11;
        float x = s->x[p] + dt * u;
        float y = s->y[p] + dt * w;
        keep_inside(&x, &u, nx);
        keep_inside(&y, &w, ny);
        s->x[p] = x; s->y[p] = y; s->u[p] = u; s->v[p] = w;
        s->c00[p] = c00; s->c01[p] = c01; s->c10[p] = c10; s->c11[p] = c11;
        float j = s->j[p] * (1.0f + dt * (c00 + c11));
        if (relax && density > OR_RELAX_MIN_DENSITY * params[P_RHO0]) {   /* Flip.java:538-543 */
            float measured = params[P_RHO0] / density;
            j = j + (params[OR_P_RELAX] * dt) * (measured - j);
        }
        s->j[p] = clampf(j, 1.0f / J_BOUND, J_BOUND);
    }
}

void or_flip2_advect(or_flip2* s, const float* params) { advect2(s, params, 0); }

void or_flip2_advect_relaxing(or_flip2* s, const float* params) { advect2(s, params, 1); }

void or_flip2_step(or_flip2* s, const float* params, or_physics ph) {   /* FlipStep.java:127-169 */
    or_flip2_clear(s);
    or_flip2_scatter(s, params, ph);
    or_flip2_grid(s, params, ph);
    or_flip2_advect(s, params);
}

void or_flip2_step_relaxing(or_flip2* s, const float* params, or_physics ph) {   /* FlipStep.java:163-166 */
    or_flip2_clear(s);
    or_flip2_scatter(s, params, ph);
    or_flip2_grid(s, params, ph);
    or_flip2_advect_relaxing(s, params);
}

/* ------------------------------------------------------------------ the sort by cell */

int32_t or_cell2(float x, float y, int nx, int ny) {                  /* Scatter.java:473-477, 535-541 */
    float cx = clampf(x, 0.0f, (float)nx - 1.0f);
    float cy = clampf(y, 0.0f, (float)ny - 1.0f);
    return (int32_t)fminf(cy, (float)(ny - 2)) * (nx - 1) + (int32_t)fminf(cx, (float)(nx - 2));
}

void or_sort2_keys(const float* x, const float* y, int64_t np, int nx, int ny, int32_t* keys) {
    for (int64_t p = 0; p < np; p++) keys[p] = or_cell2(x[p], y[p], nx, ny);
}

/* The counting sort of FlipStep.sort (count -> scan -> permute), with the order within a
 * cell defined as the order of the input (stable). The reference's atomic ranks leave that
 * order free (SortTest.java:121-134); this definition is what the device reproduces. */
void or_counting_sort(const int32_t* keys, int64_t np, int64_t cells, int32_t* starts, int32_t* perm) {
    memset(starts, 0, (size_t)(cells + 1) * sizeof(int32_t));
    for (int64_t p = 0; p < np; p++) starts[keys[p] + 1]++;
    for (int64_t c = 0; c < cells; c++) starts[c + 1] += starts[c];
    int32_t* next = (int32_t*)malloc((size_t)cells * sizeof(int32_t));
    memcpy(next, starts, (size_t)cells * sizeof(int32_t));
    for (int64_t p = 0; p < np; p++) perm[next[keys[p]]++] = (int32_t)p;
    free(next);
}

void or_apply_perm(float** fields, int nf, const int32_t* perm, int64_t np, float* tmp) {
    for (int f = 0; f < nf; f++) {
        for (int64_t d = 0; d < np; d++) tmp[d] = fields[f][perm[d]];
        memcpy(fields[f], tmp, (size_t)np * sizeof(float));
    }
}

void or_flip2_sort(or_flip2* s, int32_t* starts, int32_t* perm_scratch, float* tmp) {
    int64_t cells = (int64_t)(s->nx - 1) * (s->ny - 1);
    int32_t* keys = (int32_t*)malloc((size_t)s->np * sizeof(int32_t));
    or_sort2_keys(s->x, s->y, s->np, s->nx, s->ny, keys);
    or_counting_sort(keys, s->np, cells, starts, perm_scratch);
    float* fields[10] = {s->x, s->y, s->u, s->v, s->m, s->j, s->c00, s->c01, s->c10, s->c11};
    or_apply_perm(fields, 10, perm_scratch, s->np, tmp);
    free(keys);
}

int32_t or_cell_starts2(const float* x, const float* y, int64_t np, int nx, int ny, int32_t* starts, int64_t* bad) {
    int64_t cells = (int64_t)(nx - 1) * (ny - 1);                     /* Scatter.java:484-502 */
    memset(starts, 0, (size_t)(cells + 1) * sizeof(int32_t));
    int32_t previous = 0;
    for (int64_t p = 0; p < np; p++) {
        int32_t c = or_cell2(x[p], y[p], nx, ny);
        if (c < previous) { if (bad) *bad = p; return -1; }
        previous = c;
        starts[c + 1]++;
    }
    for (int64_t c = 0; c < cells; c++) starts[c + 1] += starts[c];
    return 0;
}

/* ------------------------------------------------------------------ bilinear P2G */

/* Scatter.Cell.of / Particle.load / deposit (Scatter.java:535-596), in particle order. */
void or_scatter2_bilinear(int nx, int ny, const float* x, const float* y, const float* u, const float* v,
                          const float* m, int64_t np, float* gm, float* gmu, float* gmv) {
    memset(gm, 0, (size_t)nx * ny * sizeof(float));
    memset(gmu, 0, (size_t)nx * ny * sizeof(float));
    memset(gmv, 0, (size_t)nx * ny * sizeof(float));
    for (int64_t p = 0; p < np; p++) {
        float cx = clampf(x[p], 0.0f, (float)nx - 1.0f);
        float cy = clampf(y[p], 0.0f, (float)ny - 1.0f);
        int col = (int)fminf(cx, (float)(nx - 2));
        int row = (int)fminf(cy, (float)(ny - 2));
        float fx = cx - (float)col;
        float fy = cy - (float)row;
        int corner = row * nx + col;
        for (int k = 0; k < 4; k++) {
            float wx = (k & 1) ? fx : 1.0f - fx;
            float wy = (k >> 1) ? fy : 1.0f - fy;
            float w = wx * wy;
            float wm = w * m[p];
            int node = corner + (k >> 1) * nx + (k & 1);
            gm[node] += wm;
            gmu[node] += wm * u[p];
            gmv[node] += wm * v[p];
        }
    }
}

/* ScatterTest.reference (ScatterTest.java:429-451): the deposit in double precision. */
void or_scatter2_bilinear_f64(int nx, int ny, const float* x, const float* y, const float* u, const float* v,
                              const float* m, int64_t np, double* gm, double* gmu, double* gmv) {
    memset(gm, 0, (size_t)nx * ny * sizeof(double));
    memset(gmu, 0, (size_t)nx * ny * sizeof(double));
    memset(gmv, 0, (size_t)nx * ny * sizeof(double));
    for (int64_t p = 0; p < np; p++) {
        double xx = fmin(fmax((double)x[p], 0.0), (double)(nx - 1));
        double yy = fmin(fmax((double)y[p], 0.0), (double)(ny - 1));
        int col = (int)fmin(xx, (double)(nx - 2));
        int row = (int)fmin(yy, (double)(ny - 2));
        double fx = xx - col, fy = yy - row, mm = m[p];
        for (int k = 0; k < 4; k++) {
            int east = k & 1, north = k >> 1;
            double w = (east ? fx : 1 - fx) * (north ? fy : 1 - fy);
            int node = (row + north) * nx + col + east;
            gm[node] += w * mm;
            gmu[node] += w * mm * u[p];
            gmv[node] += w * mm * v[p];
        }
    }
}

/* FixedScatter.kernel with its Quanta (FixedScatter.java:153-229): exact in any order. */
void or_fixed_scatter2(int nx, int ny, const float* x, const float* y, const float* u, const float* v,
                       const float* m, int64_t np, int mass_bits, int velocity_bits,
                       int32_t* gm, int32_t* gmu, int32_t* gmv) {
    const int ONE = 1 << 10;
    const float mscale = ldexpf(1.0f, mass_bits), vscale = ldexpf(1.0f, velocity_bits);
    memset(gm, 0, (size_t)nx * ny * sizeof(int32_t));
    memset(gmu, 0, (size_t)nx * ny * sizeof(int32_t));
    memset(gmv, 0, (size_t)nx * ny * sizeof(int32_t));
    for (int64_t p = 0; p < np; p++) {
        float cx = clampf(x[p], 0.0f, (float)nx - 1.0f);
        float cy = clampf(y[p], 0.0f, (float)ny - 1.0f);
        int col = (int)fminf(cx, (float)(nx - 2));
        int row = (int)fminf(cy, (float)(ny - 2));
        float fx = cx - (float)col, fy = cy - (float)row;
        int corner = row * nx + col;
        int32_t mass = (int32_t)(m[p] * mscale);
        int32_t uq = (int32_t)(u[p] * vscale), vq = (int32_t)(v[p] * vscale);
        int32_t ox = (int32_t)(fx * (float)ONE), oy = (int32_t)(fy * (float)ONE);
        int32_t high = mass / ONE, low = mass % ONE, left = mass;
        int32_t shares[4];
        for (int k = 0; k < 3; k++) {
            int32_t ax = (k & 1) ? ox : ONE - ox;
            int32_t ay = (k >> 1) ? oy : ONE - oy;
            int32_t q = ax * ay;
            int32_t share = (q * high + (q * low) / ONE) / ONE;
            left -= share;
            shares[k] = share;
        }
        shares[3] = left;
        for (int k = 0; k < 4; k++) {
            int node = corner + (k >> 1) * nx + (k & 1);
            gm[node] = (int32_t)((uint32_t)gm[node] + (uint32_t)shares[k]);
            gmu[node] = (int32_t)((uint32_t)gmu[node] + (uint32_t)shares[k] * (uint32_t)uq);
            gmv[node] = (int32_t)((uint32_t)gmv[node] + (uint32_t)shares[k] * (uint32_t)vq);
        }
    }
}
