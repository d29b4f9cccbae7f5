/*
 * tension3.c -- surface tension for the 3D step (particle/Tension3.java) restated in C: the node mass to a colour,
 * its [1 2 1]^3/64 blurs, the capillary stress, and the stress's flux across a node's faces.
 *
 * Test infrastructure only (see oracle.h). Operand order follows the IR; paths are relative to
 * vexelray-sim-fluid-core/src/main/java/dev/vexelray/sim/fluid/. Built with -ffp-contract=off, so each
 * operation rounds once, as the reference's f32 arithmetic does. The node loops are independent per node, so
 * their OpenMP split changes no bit.
 */
#include "oracle.h"
#include <math.h>
#include <stdlib.h>

enum { P_RHO0 = 5 };
static const int LOW = 1;                                 /* (int) Flip3.WALL, Tension3.java:94 */
static const float EPS2 = (float)(1e-4 * 1e-4);           /* f(EPS * EPS), Tension3.java:57, 145 */

/* Tension3.held (Tension3.java:219-221): clamp(coordinate + offset, WALL, size - 1 - WALL) as an int. The
 * reference clamps in float; every value here is a small integer, exact in float, so the integer clamp is the same. */
static inline int held(int c, int offset, int size) {
    int v = c + offset;
    return v < LOW ? LOW : v > size - 1 - LOW ? size - 1 - LOW : v;
}

static inline int64_t index3(int nx, int ny, int x, int y, int z) { return ((int64_t)z * ny + y) * nx + x; }

void or_tension3_blur(int nx, int ny, int nz, const float* src, float* dst, const float* params, int scaled) {
    const int64_t nodes = (int64_t)nx * ny * nz;
    const int size[3] = {nx, ny, nz};
#pragma omp parallel for schedule(static)
    for (int64_t node = 0; node < nodes; node++) {                 /* Tension3.java:76-105 */
        const int at[3] = {(int)(node % nx), (int)((node / nx) % ny), (int)(node / ((int64_t)nx * ny))};
        float sum = 0.0f;
        for (int dk = -1; dk <= 1; dk++) {
            for (int dj = -1; dj <= 1; dj++) {
                for (int di = -1; di <= 1; di++) {
                    const float weight = (float)((2 - abs(di)) * (2 - abs(dj)) * (2 - abs(dk)) / 64.0);
                    const int d[3] = {di, dj, dk};
                    int c[3];
                    for (int a = 0; a < 3; a++) c[a] = held(at[a], d[a], size[a]);
                    float value = src[index3(nx, ny, c[0], c[1], c[2])];
                    if (scaled) {                                   /* Tension3.java:84-99 */
                        float full = params[P_RHO0];
                        for (int a = 0; a < 3; a++) {
                            if (c[a] == LOW) full = 0.5f * full;
                            if (c[a] == size[a] - 1 - LOW) full = 0.5f * full;
                        }
                        value = fminf(value / full, 1.0f);
                    }
                    sum = sum + weight * value;
                }
            }
        }
        dst[node] = sum;
    }
}

const float* or_tension3_colour(int nx, int ny, int nz, const float* gm, const float* params, float* c0,
                                float* c1) {                          /* Flip3Step.java:95-103 */
    const float* from = gm;
    for (int k = 0; k < OR_TENSION_BLURS; k++) {
        float* to = k % 2 == 0 ? c0 : c1;
        or_tension3_blur(nx, ny, nz, from, to, params, k == 0);
        from = to;
    }
    return from;
}

void or_tension3_stress(int nx, int ny, int nz, const float* colour, float* stress) {
    const int64_t nodes = (int64_t)nx * ny * nz;
    const int size[3] = {nx, ny, nz};
#pragma omp parallel for schedule(static)
    for (int64_t node = 0; node < nodes; node++) {                 /* Tension3.java:131-152 */
        const int at[3] = {(int)(node % nx), (int)((node / nx) % ny), (int)(node / ((int64_t)nx * ny))};
        float g[3];
        for (int a = 0; a < 3; a++) {
            int up[3] = {0, 0, 0}, down[3] = {0, 0, 0};
            up[a] = 1;
            down[a] = -1;
            float hi = colour[index3(nx, ny, held(at[0], up[0], size[0]), held(at[1], up[1], size[1]),
                                     held(at[2], up[2], size[2]))];
            float lo = colour[index3(nx, ny, held(at[0], down[0], size[0]), held(at[1], down[1], size[1]),
                                     held(at[2], down[2], size[2]))];
            g[a] = 0.5f * (hi - lo);
        }
        float xx = g[0] * g[0], yy = g[1] * g[1], zz = g[2] * g[2];
        float length = sqrtf((xx + (yy + zz)) + EPS2);
        stress[0 * nodes + node] = (yy + zz) / length;
        stress[1 * nodes + node] = (xx + zz) / length;
        stress[2 * nodes + node] = (xx + yy) / length;
        stress[3 * nodes + node] = -((g[0] * g[1]) / length);
        stress[4 * nodes + node] = -((g[0] * g[2]) / length);
        stress[5 * nodes + node] = -((g[1] * g[2]) / length);
    }
}

void or_tension3_force(int nx, int ny, int nz, const float* colour, const float* stress, const int at[3],
                       float force[3]) {
    const int64_t nodes = (int64_t)nx * ny * nz;
    const int size[3] = {nx, ny, nz};
    /* the stress component a face along axis a carries for force component c (Tension3.java:163-166) */
    static const int tensor[3][3] = {{0, 3, 4}, {3, 1, 5}, {4, 5, 2}};
    const int64_t self = index3(nx, ny, at[0], at[1], at[2]);
    force[0] = force[1] = force[2] = 0.0f;
    int ring = colour[self] > OR_MIN_COLOUR;                       /* Tension3.java:172-176 */
    for (int a = 0; a < 3; a++) ring = ring && !(at[a] < LOW) && !(at[a] > size[a] - 1 - LOW);
    for (int a = 0; a < 3; a++) {
        for (int sign = -1; sign <= 1; sign += 2) {                /* Tension3.java:177-198 */
            int d[3] = {0, 0, 0};
            d[a] = sign;
            const int64_t there = index3(nx, ny, held(at[0], d[0], size[0]), held(at[1], d[1], size[1]),
                                         held(at[2], d[2], size[2]));
            const int open = ring && colour[there] > OR_MIN_COLOUR;
            const int wall = sign < 0 ? !(at[a] > LOW) : !(at[a] < size[a] - 1 - LOW);
            const float shear = wall ? 0.0f : 1.0f;
            if (!open) continue;
            for (int c = 0; c < 3; c++) {
                const float* t = stress + (int64_t)tensor[a][c] * nodes;
                float flux = (0.5f * (float)sign) * (t[self] + t[there]);
                force[c] = force[c] + (c == a ? flux : shear * flux);
            }
        }
    }
}
