/*
 * mpm3.c -- the 3D MLS-MPM/APIC step (Flip3.java) restated in C, plus the 3D sort
 * by stencil cell that the reference does not have (Flip3.java:44-48 and
 * Flip3Step.java:17-20 leave the 3D particles unsorted; docs/TODO.md:191-197
 * proposes the sort by stencil this defines).
 *
 * Test infrastructure only (see oracle.h). Operand order follows the IR;
 * paths are relative to vexelray-sim-fluid-core/src/main/java/dev/vexelray/sim/fluid/.
 */
#include "oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

static inline float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

/* particle/Flip3.java:58-64 */
enum { P_DT = 0, P_GX = 1, P_GY = 2, P_GZ = 3, P_BULK = 4, P_RHO0 = 5 };
static const float WALL = 1.0f;          /* Flip3.java:67 */
static const int WALL_NODE = 1;          /* Flip3.java:68 */
static const float EMPTY = 1e-9f;        /* Flip3.java:71 */
static const float J_BOUND = 10.0f;      /* Flip3.java:74 */

static inline float impulse(float dt, float m, float rho0, float bulk, float j, int eos) {
    float jp;
    if (eos == OR_EOS_TAIT) {
        float r = 1.0f / j;
        float r2 = r * r;
        float r6 = (r2 * r2) * r2;
        jp = bulk * (r6 - j);
    } else {
        jp = bulk * (1.0f - j);                                   /* Flip3.java:216-218 */
    }
    return (4.0f * (dt * (m / rho0))) * jp;
}

/* Flip3.Stencil3 (Flip3.java:662-711) */
typedef struct { int cell[3]; int base; float off[3]; float w[3][3]; } stencil3;

static inline void weights(float f, float w[3]) {
    float a = 1.5f - f;
    float c = f - 1.0f;
    float e = f - 0.5f;
    w[0] = 0.5f * (a * a);
    w[1] = 0.75f - c * c;
    w[2] = 0.5f * (e * e);
}

static inline stencil3 stencil_of(float px, float py, float pz, int nx, int ny, int nz) {
    stencil3 s;
    const float at[3] = {px, py, pz};
    const int size[3] = {nx, ny, nz};
    for (int a = 0; a < 3; a++) {
        float x = clampf(at[a], 0.5f, (float)size[a] - 1.5f);
        s.cell[a] = (int)fminf(x - 0.5f, (float)(size[a] - 3));
        s.off[a] = x - (float)s.cell[a];
        weights(s.off[a], s.w[a]);
    }
    s.base = (s.cell[2] * ny + s.cell[1]) * nx + s.cell[0];
    return s;
}

static inline float weight_k(const stencil3* s, int k) {           /* Flip3.java:690-692 */
    return s->w[0][k % 3] * (s->w[1][(k / 3) % 3] * s->w[2][k / 9]);
}

static inline int offset_k(int k, int nx, int ny) {                 /* Flip3.java:708-710 */
    return (k / 9) * nx * ny + ((k / 3) % 3) * nx + k % 3;
}

void or_flip3_clear(or_flip3* s) {                                  /* Flip3.java:163-172 */
    size_t n = (size_t)s->nx * s->ny * s->nz;
    memset(s->gm, 0, n * sizeof(float));
    memset(s->gmu, 0, n * sizeof(float));
    memset(s->gmv, 0, n * sizeof(float));
    memset(s->gmw, 0, n * sizeof(float));
}

void or_flip3_scatter(or_flip3* s, const float* params, or_physics ph) {   /* Flip3.java:193-246 */
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const float dt = params[P_DT], bulk = params[P_BULK], rho0 = params[P_RHO0];
    float* grid[4] = {s->gm, s->gmu, s->gmv, s->gmw};
    for (int p = 0; p < s->np; p++) {
        if (!(s->m[p] > 0.0f)) continue;
        stencil3 st = stencil_of(s->x[p], s->y[p], s->z[p], nx, ny, nz);
        float m = s->m[p];
        float vel[3] = {s->u[p], s->v[p], s->w[p]};
        float c[9];
        for (int a = 0; a < 9; a++) c[a] = s->c[a][p];
        float sp = impulse(dt, m, rho0, bulk, s->j[p], ph.eos);
        for (int k = 0; k < 27; k++) {
            float wgt = weight_k(&st, k);
            float d[3] = {(float)(k % 3) - st.off[0], (float)((k / 3) % 3) - st.off[1], (float)(k / 9) - st.off[2]};
            float wm = wgt * m;
            int node = st.base + offset_k(k, nx, ny);
            grid[0][node] += wm;
            for (int a = 0; a < 3; a++) {
                float at3 = vel[a] + (c[3 * a] * d[0] + (c[3 * a + 1] * d[1] + c[3 * a + 2] * d[2]));
                float push = sp * d[a];
                grid[1 + a][node] += wm * at3 + wgt * push;
            }
        }
    }
}

/* The exact 3D scatter: the amounts of or_flip3_scatter (same operand order, no fused multiply-add), each
 * quantized to 2^-40 (round to nearest even) and summed as int64, so the result does not depend on the order of
 * the particles. The centre node (1,1,1) takes what the other 26 mass shares leave of the particle's quantized
 * mass. The 3D form of FixedScatter (FixedScatter.java:24-60; 64-bit sums instead of its 32-bit ones). q holds
 * four planes of nx*ny*nz values: m, mu, mv, mw; it is zeroed first. */
static inline int64_t fixed3(float v) { return (int64_t)llrintf(v * 0x1p40f); }

void or_fixed_scatter3(or_flip3* s, const float* params, or_physics ph, int64_t* q) {
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const size_t nodes = (size_t)nx * ny * nz;
    const float dt = params[P_DT], bulk = params[P_BULK], rho0 = params[P_RHO0];
    memset(q, 0, 4 * nodes * sizeof(int64_t));
    for (int p = 0; p < s->np; p++) {
        if (!(s->m[p] > 0.0f)) continue;
        stencil3 st = stencil_of(s->x[p], s->y[p], s->z[p], nx, ny, nz);
        float m = s->m[p];
        float vel[3] = {s->u[p], s->v[p], s->w[p]};
        float c[9];
        for (int a = 0; a < 9; a++) c[a] = s->c[a][p];
        float sp = impulse(dt, m, rho0, bulk, s->j[p], ph.eos);
        int64_t rest = fixed3(m);
        for (int k = 0; k < 27; k++) {
            float wgt = weight_k(&st, k);
            float d[3] = {(float)(k % 3) - st.off[0], (float)((k / 3) % 3) - st.off[1], (float)(k / 9) - st.off[2]};
            float wm = wgt * m;
            size_t node = (size_t)(st.base + offset_k(k, nx, ny));
            if (k != 13) {
                int64_t share = fixed3(wm);
                rest -= share;
                q[node] = (int64_t)((uint64_t)q[node] + (uint64_t)share);
            }
            for (int a = 0; a < 3; a++) {
                float at3 = vel[a] + (c[3 * a] * d[0] + (c[3 * a + 1] * d[1] + c[3 * a + 2] * d[2]));
                float push = sp * d[a];
                float mom = wm * at3 + wgt * push;
                q[(1 + a) * nodes + node] = (int64_t)((uint64_t)q[(1 + a) * nodes + node] + (uint64_t)fixed3(mom));
            }
        }
        size_t centre = (size_t)(st.base + offset_k(13, nx, ny));
        q[centre] = (int64_t)((uint64_t)q[centre] + (uint64_t)rest);
    }
}

static void grid3(or_flip3* s, const float* params, or_physics ph, const float* colour, const float* stress) {
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const int size[3] = {nx, ny, nz};
    const float g[3] = {params[P_GX], params[P_GY], params[P_GZ]};
    const float* mom[3] = {s->gmu, s->gmv, s->gmw};
    float* out[3] = {s->gu, s->gv, s->gw};
    int64_t nodes = (int64_t)nx * ny * nz;
#pragma omp parallel for schedule(static)   /* each node alone: the split changes no bit */
    for (int64_t node = 0; node < nodes; node++) {
        int at[3] = {(int)(node % nx), (int)((node / nx) % ny), (int)(node / ((int64_t)nx * ny))};
        float mass = s->gm[node];
        float vel[3] = {0.0f, 0.0f, 0.0f};
        if (mass > EMPTY) {
            float dt = params[P_DT];
            for (int a = 0; a < 3; a++) vel[a] = mom[a][node] / mass + dt * g[a];
            if (colour) {                                                  /* Flip3.java:291-299 */
                float force[3];
                or_tension3_force(nx, ny, nz, colour, stress, at, force);
                float push = (dt * params[6]) / fmaxf(mass, OR_MASS_FLOOR * params[P_RHO0]);
                for (int a = 0; a < 3; a++) vel[a] = vel[a] + push * force[a];
            }
        }
        int stuck = 0;
        if (ph.sticky > 0) {
            for (int a = 0; a < 3; a++) if (at[a] < ph.sticky || at[a] > size[a] - 1 - ph.sticky) stuck = 1;
        }
        for (int a = 0; a < 3; a++) {
            if (ph.sticky > 0) {
                if (stuck) vel[a] = 0.0f;
            } else {
                if (!(at[a] > WALL_NODE)) vel[a] = fmaxf(vel[a], 0.0f);
                if (at[a] > size[a] - 2 - WALL_NODE) vel[a] = fminf(vel[a], 0.0f);
            }
            out[a][node] = vel[a];
        }
    }
}

void or_flip3_grid(or_flip3* s, const float* params, or_physics ph) {      /* Flip3.java:267-311 */
    grid3(s, params, ph, NULL, NULL);
}

void or_flip3_grid_tension(or_flip3* s, const float* params, or_physics ph, const float* colour,
                           const float* stress) {                        /* Flip3.java:258-310 */
    grid3(s, params, ph, colour, stress);
}

static inline void keep_inside(float* at, float* vel, int size) {   /* Flip3.java:644-655 */
    float lo = WALL;
    float hi = (float)size - 1.0f - WALL;
    if (*at < lo) { *at = lo; *vel = fmaxf(*vel, 0.0f); }
    if (*at > hi) { *at = hi; *vel = fminf(*vel, 0.0f); }
}

void or_flip3_advect(or_flip3* s, const float* params) {           /* Flip3.java:329-383 */
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const int size[3] = {nx, ny, nz};
    const float* grid[3] = {s->gu, s->gv, s->gw};
    float* at[3] = {s->x, s->y, s->z};
    float* velocity[3] = {s->u, s->v, s->w};
    for (int p = 0; p < s->np; p++) {
        if (!(s->m[p] > 0.0f)) continue;
        stencil3 st = stencil_of(s->x[p], s->y[p], s->z[p], nx, ny, nz);
        float vel[3] = {0, 0, 0};
        float sum[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int k = 0; k < 27; k++) {
            float wgt = weight_k(&st, k);
            float d[3] = {(float)(k % 3) - st.off[0], (float)((k / 3) % 3) - st.off[1], (float)(k / 9) - st.off[2]};
            int node = st.base + offset_k(k, nx, ny);
            for (int a = 0; a < 3; a++) {
                float node_a = wgt * grid[a][node];
                vel[a] = vel[a] + node_a;
                for (int e = 0; e < 3; e++) sum[3 * a + e] = sum[3 * a + e] + node_a * d[e];
            }
        }
        float dt = params[P_DT];
        float c[9];
        for (int a = 0; a < 9; a++) c[a] = 4.0f * sum[a];
        for (int a = 0; a < 3; a++) {
            float pos = at[a][p] + dt * vel[a];
            keep_inside(&pos, &vel[a], size[a]);
            at[a][p] = pos;
            velocity[a][p] = vel[a];
        }
        for (int a = 0; a < 9; a++) s->c[a][p] = c[a];
        float j = s->j[p] * (1.0f + dt * (c[0] + (c[4] + c[8])));
        s->j[p] = clampf(j, 1.0f / J_BOUND, J_BOUND);
    }
}

void or_flip3_step(or_flip3* s, const float* params, or_physics ph) {   /* Flip3Step.java:81-118 */
    or_flip3_clear(s);
    or_flip3_scatter(s, params, ph);
    or_flip3_grid(s, params, ph);
    or_flip3_advect(s, params);
}

void or_flip3_step_tension(or_flip3* s, const float* params, or_physics ph, float* scratch) {
    const int64_t nodes = (int64_t)s->nx * s->ny * s->nz;
    or_flip3_clear(s);
    or_flip3_scatter(s, params, ph);
    const float* colour = or_tension3_colour(s->nx, s->ny, s->nz, s->gm, params, scratch, scratch + nodes);
    or_tension3_stress(s->nx, s->ny, s->nz, colour, scratch + 2 * nodes);
    or_flip3_grid_tension(s, params, ph, colour, scratch + 2 * nodes);
    or_flip3_advect(s, params);
}

/* ------------------------------------------------------------------ 3D sort key */

/* The stencil base cell of Stencil3 (Flip3.java:671-673): cell_a in [0, n_a-3]. It is
 * linearised brick-major: bricks of 8x8x8 cells, bricks in x-fastest order, and cells
 * x-fastest within a brick, so each brick's particles are one contiguous run. */
static inline void bricks3(int nx, int ny, int nz, int nb[3]) {
    nb[0] = (nx - 2 + OR_BRICK - 1) / OR_BRICK;
    nb[1] = (ny - 2 + OR_BRICK - 1) / OR_BRICK;
    nb[2] = (nz - 2 + OR_BRICK - 1) / OR_BRICK;
}

int64_t or_key3_count(int nx, int ny, int nz) {
    int nb[3];
    bricks3(nx, ny, nz, nb);
    return (int64_t)nb[0] * nb[1] * nb[2] * OR_BRICK_CELLS;
}

int32_t or_key3(float x, float y, float z, int nx, int ny, int nz) {
    int nb[3];
    bricks3(nx, ny, nz, nb);
    const float at[3] = {x, y, z};
    const int size[3] = {nx, ny, nz};
    int cell[3];
    for (int a = 0; a < 3; a++) {
        float c = clampf(at[a], 0.5f, (float)size[a] - 1.5f);
        cell[a] = (int)fminf(c - 0.5f, (float)(size[a] - 3));
    }
    int brick = ((cell[2] / OR_BRICK) * nb[1] + cell[1] / OR_BRICK) * nb[0] + cell[0] / OR_BRICK;
    int local = ((cell[2] % OR_BRICK) * OR_BRICK + cell[1] % OR_BRICK) * OR_BRICK + cell[0] % OR_BRICK;
    return brick * OR_BRICK_CELLS + local;
}

void or_flip3_sort(or_flip3* s, int32_t* starts, int32_t* keys, int32_t* perm, float* tmp) {
    int64_t nk = or_key3_count(s->nx, s->ny, s->nz);
    for (int p = 0; p < s->np; p++) keys[p] = or_key3(s->x[p], s->y[p], s->z[p], s->nx, s->ny, s->nz);
    or_counting_sort(keys, s->np, nk, starts, perm);
    float* fields[17] = {s->x, s->y, s->z, s->u, s->v, s->w, s->m, s->j,
                         s->c[0], s->c[1], s->c[2], s->c[3], s->c[4], s->c[5], s->c[6], s->c[7], s->c[8]};
    or_apply_perm(fields, 17, perm, s->np, tmp);
}

/* ------------------------------------------------------------------ threaded step (CPU baseline) */

#ifdef _OPENMP
#include <omp.h>
#endif

int or_baseline_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* The same step with the particle loops threaded: each thread scatters its slice of the
 * particles into a private grid, over only the z-planes its slice touches, and the private
 * grids are summed plane by plane. Grid update and advect are plain parallel loops. The
 * arithmetic per particle and per node is that of the sequential functions above. */
static void step_omp(or_flip3* s, const float* params, or_physics ph, float* scratch, float* tension) {
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const int64_t plane = (int64_t)nx * ny, nodes = plane * nz;
    const float dt = params[P_DT], bulk = params[P_BULK], rho0 = params[P_RHO0];
    int nt = or_baseline_threads();
    /* Private grids: one per thread, allocated once and touched only on the z-planes each thread's
     * particles reach, so only those pages are ever backed. */
    static float* own = NULL;
    static size_t own_floats = 0;
    if (!scratch) {
        size_t want = (size_t)nt * 4 * (size_t)nodes;
        if (own_floats < want) {
            free(own);
            own = (float*)malloc(want * sizeof(float));
            own_floats = own ? want : 0;
        }
        scratch = own;
        if (!scratch) return;
    }
    int zlo[256], zhi[256];
    if (nt > 256) nt = 256;
#pragma omp parallel num_threads(nt)
    {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        float* g = scratch + (size_t)t * 4 * nodes;
        int64_t p0 = (int64_t)s->np * t / nt, p1 = (int64_t)s->np * (t + 1) / nt;
        int lo = nz, hi = -1;
        for (int64_t p = p0; p < p1; p++) {
            if (!(s->m[p] > 0.0f)) continue;
            stencil3 st = stencil_of(s->x[p], s->y[p], s->z[p], nx, ny, nz);
            if (st.cell[2] < lo) lo = st.cell[2];
            if (st.cell[2] + 2 > hi) hi = st.cell[2] + 2;
        }
        zlo[t] = lo; zhi[t] = hi;
        if (hi >= lo) memset(g + (size_t)lo * plane * 4, 0, (size_t)(hi - lo + 1) * plane * 4 * sizeof(float));
        for (int64_t p = p0; p < p1; p++) {
            if (!(s->m[p] > 0.0f)) continue;
            stencil3 st = stencil_of(s->x[p], s->y[p], s->z[p], nx, ny, nz);
            float m = s->m[p];
            float vel[3] = {s->u[p], s->v[p], s->w[p]};
            float c[9];
            for (int a = 0; a < 9; a++) c[a] = s->c[a][p];
            float sp = impulse(dt, m, rho0, bulk, s->j[p], ph.eos);
            for (int k = 0; k < 27; k++) {
                float wgt = weight_k(&st, k);
                float d[3] = {(float)(k % 3) - st.off[0], (float)((k / 3) % 3) - st.off[1], (float)(k / 9) - st.off[2]};
                float wm = wgt * m;
                int64_t node = st.base + offset_k(k, nx, ny);
                float* q = g + (size_t)node * 4;
                q[0] += wm;
                for (int a = 0; a < 3; a++) {
                    float at3 = vel[a] + (c[3 * a] * d[0] + (c[3 * a + 1] * d[1] + c[3 * a + 2] * d[2]));
                    q[1 + a] += wm * at3 + wgt * (sp * d[a]);
                }
            }
        }
#pragma omp barrier
        /* sum the private grids, plane by plane, planes split across threads */
#pragma omp for schedule(static)
        for (int z = 0; z < nz; z++) {
            float* gm = s->gm + z * plane; float* gu = s->gmu + z * plane;
            float* gv = s->gmv + z * plane; float* gw = s->gmw + z * plane;
            memset(gm, 0, plane * sizeof(float)); memset(gu, 0, plane * sizeof(float));
            memset(gv, 0, plane * sizeof(float)); memset(gw, 0, plane * sizeof(float));
            for (int u = 0; u < nt; u++) {
                if (z < zlo[u] || z > zhi[u]) continue;
                const float* q = scratch + (size_t)u * 4 * nodes + (size_t)z * plane * 4;
                for (int64_t i = 0; i < plane; i++) {
                    gm[i] += q[4 * i]; gu[i] += q[4 * i + 1]; gv[i] += q[4 * i + 2]; gw[i] += q[4 * i + 3];
                }
            }
        }
    }
    /* grid update and advect: independent per node / per particle */
    const int size[3] = {nx, ny, nz};
    const float gr[3] = {params[P_GX], params[P_GY], params[P_GZ]};
    if (tension) {   /* Flip3Step with tension: the colour, its blurs, the stress, the grid with the force */
        const float* colour = or_tension3_colour(nx, ny, nz, s->gm, params, tension, tension + nodes);
        or_tension3_stress(nx, ny, nz, colour, tension + 2 * nodes);
        or_flip3_grid_tension(s, params, ph, colour, tension + 2 * nodes);
    }
#pragma omp parallel for schedule(static) num_threads(nt)
    for (int64_t node = 0; node < (tension ? 0 : nodes); node++) {
        int at[3] = {(int)(node % nx), (int)((node / nx) % ny), (int)(node / plane)};
        float mass = s->gm[node];
        float vel[3] = {0.0f, 0.0f, 0.0f};
        const float* mom[3] = {s->gmu, s->gmv, s->gmw};
        if (mass > EMPTY) for (int a = 0; a < 3; a++) vel[a] = mom[a][node] / mass + dt * gr[a];
        int stuck = 0;
        if (ph.sticky > 0) for (int a = 0; a < 3; a++) if (at[a] < ph.sticky || at[a] > size[a] - 1 - ph.sticky) stuck = 1;
        for (int a = 0; a < 3; a++) {
            if (ph.sticky > 0) { if (stuck) vel[a] = 0.0f; }
            else {
                if (!(at[a] > WALL_NODE)) vel[a] = fmaxf(vel[a], 0.0f);
                if (at[a] > size[a] - 2 - WALL_NODE) vel[a] = fminf(vel[a], 0.0f);
            }
        }
        s->gu[node] = vel[0]; s->gv[node] = vel[1]; s->gw[node] = vel[2];
    }
    or_flip3 part = *s;
#pragma omp parallel num_threads(nt)
    {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        int64_t p0 = (int64_t)s->np * t / nt, p1 = (int64_t)s->np * (t + 1) / nt;
        or_flip3 mine = part;
        mine.x += p0; mine.y += p0; mine.z += p0; mine.u += p0; mine.v += p0; mine.w += p0;
        mine.m += p0; mine.j += p0;
        for (int a = 0; a < 9; a++) mine.c[a] += p0;
        mine.np = (int)(p1 - p0);
        or_flip3_advect(&mine, params);
    }
}

void or_flip3_step_omp(or_flip3* s, const float* params, or_physics ph, float* scratch) {
    step_omp(s, params, ph, scratch, NULL);
}

void or_flip3_step_tension_omp(or_flip3* s, const float* params, or_physics ph, float* scratch, float* tension) {
    step_omp(s, params, ph, scratch, tension);
}
