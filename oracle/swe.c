/*
 * swe.c -- one dispatch of the shallow-water step (ShallowWater.java) restated in C,
 * plus the host-side fastestWave and the Diagnostics / ParticleDiagnostics readouts.
 *
 * Test infrastructure only (see oracle.h). Operand order follows the IR; paths are
 * relative to vexelray-sim-fluid-core/src/main/java/dev/vexelray/sim/fluid/.
 *
 * The kernel's two atomics are restated by their sequential meaning: CLAMPED counts
 * the cells whose raw depth was negative (ShallowWater.java:219), and SPEED_OUT ends
 * as the max of its entry value and every cell's speed bits (230-235), a max over
 * non-negative floats' bit patterns.
 */
#include "oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct { float h, hu, hv; } state;
typedef struct { float mass, normal, tangent; } flux;

static inline float bits_to_float(int32_t b) { float f; memcpy(&f, &b, 4); return f; }
static inline int32_t float_to_bits(float f) { int32_t b; memcpy(&b, &f, 4); return b; }

/* ShallowWater.velocity (329-333) */
static inline float velocity(float h, float q, float dry) { return h > dry ? q / h : 0.0f; }

/* ShallowWater.combine (381-384) */
static inline float combine(float hi, float lo, float lohi, float span, float fl, float fr, float ul, float ur) {
    return ((hi * fl - lo * fr) + lohi * (ur - ul)) / span;
}

/* ShallowWater.hll (336-378) */
static flux hll(float g, float dry, state L, state R, int normal_is_x) {
    float qnL = normal_is_x ? L.hu : L.hv;
    float qtL = normal_is_x ? L.hv : L.hu;
    float qnR = normal_is_x ? R.hu : R.hv;
    float qtR = normal_is_x ? R.hv : R.hu;
    float unL = velocity(L.h, qnL, dry);
    float utL = velocity(L.h, qtL, dry);
    float unR = velocity(R.h, qnR, dry);
    float utR = velocity(R.h, qtR, dry);
    float cL = sqrtf(g * L.h);
    float cR = sqrtf(g * R.h);
    float sL = fminf(unL - cL, unR - cR);
    float sR = fmaxf(unL + cL, unR + cR);
    if (!(R.h > dry)) { sL = unL - cL; sR = unL + 2.0f * cL; }
    if (!(L.h > dry)) { sL = unR - 2.0f * cR; sR = unR + cR; }
    float lo = fminf(sL, 0.0f);
    float hi = fmaxf(sR, 0.0f);
    float span = fmaxf(hi - lo, 1e-30f);
    float lohi = lo * hi;
    float pL = (0.5f * g) * (L.h * L.h);
    float pR = (0.5f * g) * (R.h * R.h);
    flux f;
    f.mass = combine(hi, lo, lohi, span, qnL, qnR, L.h, R.h);
    f.normal = combine(hi, lo, lohi, span, qnL * unL + pL, qnR * unR + pR, qnL, qnR);
    f.tangent = combine(hi, lo, lohi, span, qnL * utL, qnR * utR, qtL, qtR);
    return f;
}

/* ShallowWater.neighbour (316-326): the ghost at an edge is the edge cell, its normal
 * momentum negated for a wall. */
static inline state neighbour(const float* h, const float* hu, const float* hv, int cell, int at_edge,
                              int offset, int edge, int normal_is_x) {
    int index = at_edge ? cell : cell + offset;
    state s = {h[index], hu[index], hv[index]};
    if (edge == OR_EDGE_WALL && at_edge) {
        if (normal_is_x) s.hu = -s.hu; else s.hv = -s.hv;
    }
    return s;
}

static void swe_range(int nx, int ny, const int32_t edges[4], const float* params,
                      const float* in_h, const float* in_hu, const float* in_hv,
                      float* out_h, float* out_hu, float* out_hv,
                      const int32_t* speed_in, const int32_t* budget_in,
                      int64_t first, int64_t last, int32_t* max_bits, int32_t* clamps, int32_t* ticks_out) {
    const float g = params[0], courant = params[1], dx = params[2], dy = params[3], dry = params[4];
    /* ShallowWater.java:184-192: the step from the fastest wave, in whole ticks, within the budget */
    float fastest = bits_to_float(speed_in[0]);
    float allowed = fminf((courant * fminf(dx, dy)) / fmaxf(fastest, 1e-30f), 2000.0f);
    int32_t ticks = (int32_t)(allowed * 1000000.0f);
    int32_t budget = budget_in[0];
    if (budget < ticks) ticks = budget;
    float dt = (float)ticks * (float)(1.0 / 1000000.0);
    float rx = dt / dx;
    float ry = dt / dy;
    int32_t mb = *max_bits, cl = 0;
    for (int64_t c = first; c < last; c++) {
        int cell = (int)c;
        int x = cell % nx;
        int y = cell / nx;
        state here = {in_h[cell], in_hu[cell], in_hv[cell]};
        state west = neighbour(in_h, in_hu, in_hv, cell, x == 0, -1, edges[0], 1);
        state east = neighbour(in_h, in_hu, in_hv, cell, x == nx - 1, 1, edges[1], 1);
        state south = neighbour(in_h, in_hu, in_hv, cell, y == 0, -nx, edges[2], 0);
        state north = neighbour(in_h, in_hu, in_hv, cell, y == ny - 1, nx, edges[3], 0);
        flux fw = hll(g, dry, west, here, 1);
        flux fe = hll(g, dry, here, east, 1);
        flux fs = hll(g, dry, south, here, 0);
        flux fn = hll(g, dry, here, north, 0);
        float h = (here.h - rx * (fe.mass - fw.mass)) - ry * (fn.mass - fs.mass);
        float hu = (here.hu - rx * (fe.normal - fw.normal)) - ry * (fn.tangent - fs.tangent);
        float hv = (here.hv - rx * (fe.tangent - fw.tangent)) - ry * (fn.normal - fs.normal);
        if (h < 0.0f) cl++;
        float nh = fmaxf(h, 0.0f);
        out_h[cell] = nh;
        out_hu[cell] = hu;
        out_hv[cell] = hv;
        float u = velocity(nh, hu, dry);
        float w = velocity(nh, hv, dry);
        float speed = fmaxf(fabsf(u), fabsf(w)) + sqrtf(g * nh);
        int32_t sb = float_to_bits(speed);
        if (sb > mb) mb = sb;
    }
    *max_bits = mb;
    *clamps = cl;
    *ticks_out = ticks;
}

void or_swe_dispatch(int nx, int ny, const int32_t edges[4], const float* params,
                     const float* in_h, const float* in_hu, const float* in_hv,
                     float* out_h, float* out_hu, float* out_hv,
                     const int32_t* speed_in, int32_t* speed_out, int32_t* speed_clear,
                     const int32_t* budget_in, int32_t* budget_out, int32_t* clamped) {
    int32_t mb = speed_out[0], cl = 0, ticks = 0;
    int32_t budget = budget_in[0];
    swe_range(nx, ny, edges, params, in_h, in_hu, in_hv, out_h, out_hu, out_hv, speed_in, budget_in,
              0, (int64_t)nx * ny, &mb, &cl, &ticks);
    speed_out[0] = mb;
    clamped[0] += cl;
    speed_clear[0] = 0;                                   /* ShallowWater.java:237-240 */
    budget_out[0] = budget - ticks;
}

int32_t or_swe_fastest_wave(const float* h, const float* hu, const float* hv, int64_t n, double g, double dry) {
    float fastest = 0.0f;                                 /* ShallowWater.java:287-295 */
    for (int64_t k = 0; k < n; k++) {
        float u = (double)h[k] > dry ? hu[k] / h[k] : 0.0f;
        float w = (double)h[k] > dry ? hv[k] / h[k] : 0.0f;
        float c = (float)sqrt(g * (double)h[k]);
        float s = fmaxf(fabsf(u), fabsf(w)) + c;
        /* Math.max(float, float): NaN if either is NaN */
        if (isnan(s) || isnan(fastest)) fastest = NAN; else fastest = fastest > s ? fastest : s;
    }
    return float_to_bits(fastest);
}

/* ------------------------------------------------------------------ diagnostics */

void or_swe_diagnostics(const float* h, const float* hu, const float* hv, int64_t n, double g, double dry,
                        double dt, double dx, double dy, or_swe_diag* out) {   /* Diagnostics.java:43-81 */
    double volume = 0, min_depth = INFINITY, max_depth = 0, max_speed = 0, max_froude = 0, max_wave = 0;
    int32_t non_finite = 0, negative = 0, wet = 0;
    for (int64_t k = 0; k < n; k++) {
        if (!isfinite(h[k]) || !isfinite(hu[k]) || !isfinite(hv[k])) { non_finite++; continue; }
        if (h[k] < 0) negative++;
        volume += h[k];
        max_depth = fmax(max_depth, h[k]);
        if ((double)h[k] <= dry) continue;
        wet++;
        min_depth = fmin(min_depth, h[k]);
        double u = (double)hu[k] / h[k];
        double v = (double)hv[k] / h[k];
        double c = sqrt(g * h[k]);
        double speed = sqrt(u * u + v * v);
        max_speed = fmax(max_speed, speed);
        if (h[k] >= 1e-3) max_froude = fmax(max_froude, speed / c);
        max_wave = fmax(max_wave, fmax(fabs(u), fabs(v)) + c);
    }
    out->volume = volume * dx * dy;
    out->min_depth = wet == 0 ? 0 : min_depth;
    out->max_depth = max_depth;
    out->max_speed = max_speed;
    out->max_froude = max_froude;
    out->max_courant = max_wave * dt / fmin(dx, dy);
    out->non_finite = non_finite;
    out->negative = negative;
    out->wet = wet;
}

static int cmp_float(const void* a, const void* b) {
    float x = *(const float*)a, y = *(const float*)b;
    return (x > y) - (x < y);
}

void or_particle_diagnostics(const float* j, int64_t n, double speed, double sound, double dt,
                             or_particle_diag* out) {   /* ParticleDiagnostics.java:126-148 */
    float* valid = (float*)malloc((size_t)(n > 0 ? n : 1) * sizeof(float));
    int64_t m = 0;
    for (int64_t k = 0; k < n; k++) if (isfinite(j[k]) && j[k] > 0) valid[m++] = j[k];
    out->non_finite = (int32_t)(n - m);
    out->mach = speed / sound;
    out->courant = (speed + sound) * dt;
    if (m == 0) {
        out->min_density = out->max_density = out->low_density = out->high_density = 0;
        free(valid);
        return;
    }
    qsort(valid, (size_t)m, sizeof(float), cmp_float);
    int64_t p99 = (int64_t)(0.99 * m); if (p99 > m - 1) p99 = m - 1;
    int64_t p01 = (int64_t)(0.01 * m); if (p01 > m - 1) p01 = m - 1;
    /* Java's 1 / valid[k] with valid a float[] is a float division (the int 1 is promoted to float); the
       record's double field then holds the float quotient */
    out->min_density = (double)(1.0f / valid[m - 1]);
    out->max_density = (double)(1.0f / valid[0]);
    out->low_density = (double)(1.0f / valid[p99]);
    out->high_density = (double)(1.0f / valid[p01]);
    free(valid);
}

/* ------------------------------------------------------------------ threaded SWE (CPU baseline) */

#ifdef _OPENMP
#include <omp.h>
#endif

void or_swe_dispatch_omp(int nx, int ny, const int32_t edges[4], const float* params,
                         const float* in_h, const float* in_hu, const float* in_hv,
                         float* out_h, float* out_hu, float* out_hv,
                         const int32_t* speed_in, int32_t* speed_out, int32_t* speed_clear,
                         const int32_t* budget_in, int32_t* budget_out, int32_t* clamped) {
    int32_t mb_all = speed_out[0], cl_all = 0, ticks_all = 0;
    int32_t budget = budget_in[0];
#pragma omp parallel
    {
        int nt = 1, t = 0;
#ifdef _OPENMP
        nt = omp_get_num_threads();
        t = omp_get_thread_num();
#endif
        int64_t rows = ny, r0 = rows * t / nt, r1 = rows * (t + 1) / nt;
        int32_t mb = mb_all, cl = 0, ticks = 0;
        swe_range(nx, ny, edges, params, in_h, in_hu, in_hv, out_h, out_hu, out_hv, speed_in, budget_in,
                  r0 * nx, r1 * nx, &mb, &cl, &ticks);
#pragma omp critical
        {
            if (mb > mb_all) mb_all = mb;
            cl_all += cl;
            ticks_all = ticks;
        }
    }
    speed_out[0] = mb_all;
    clamped[0] += cl_all;
    speed_clear[0] = 0;
    budget_out[0] = budget - ticks_all;
}
