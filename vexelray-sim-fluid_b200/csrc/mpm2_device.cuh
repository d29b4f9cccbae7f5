// mpm2_device.cuh -- the 2D MLS-MPM/APIC step's per-particle and per-node arithmetic (Flip.java),
// shared by the single-scene step (mpm2.cu) and the batched scenes (batch2.cu). Every operation
// keeps the reference's operand order; the rounding-sensitive ones are written as _rn intrinsics
// so no contraction changes them.
#pragma once

#include "common.cuh"

namespace vf {

enum Field2 { PX = 0, PY, PU, PV, PM, PJ, PC00, PC01, PC10, PC11, NF2 };

// Device copy of Flip.params' first five words (Flip.java:145-211) plus the physics options.
struct Params2 {
    float dt, gx, gy, bulk, rho0;
    int tait, sticky;
    float relax;     // Flip.params' RELAX word (Flip.java:113): J's pull toward the mass's volume, per second
    int relaxing;    // VF_RELAX: the step's advect is Flip.advectRelaxing
};

constexpr float EMPTY2 = 1e-9f;     // Flip.java:316
constexpr float J_BOUND2 = 10.0f;   // Flip.java:430
constexpr float RELAX_MIN_DENSITY2 = 0.8f;   // Flip.java:449

// Flip.Stencil.of (Flip.java:572-581): the lower-left node of the 3x3 stencil, the offsets in
// [1/2, 3/2] and the quadratic B-spline weights per axis.
struct Stencil2 {
    int col, row, base;
    float fx, fy, wx[3], wy[3];
};

__device__ __forceinline__ Stencil2 stencil2(float px, float py, int nx, int ny) {
    Stencil2 s;
    float x = clampf(px, 0.5f, (float)nx - 1.5f);
    float y = clampf(py, 0.5f, (float)ny - 1.5f);
    s.col = (int)fminf(__fsub_rn(x, 0.5f), (float)(nx - 3));
    s.row = (int)fminf(__fsub_rn(y, 0.5f), (float)(ny - 3));
    s.fx = __fsub_rn(x, (float)s.col);
    s.fy = __fsub_rn(y, (float)s.row);
    s.base = s.row * nx + s.col;
    bspline_weights(s.fx, s.wx);
    bspline_weights(s.fy, s.wy);
    return s;
}

// The stencil's lower-left node alone (the batched sort's cell), as stencil2 computes it.
__device__ __forceinline__ void stencil_cell2(float px, float py, int nx, int ny, int& col, int& row) {
    float x = clampf(px, 0.5f, (float)nx - 1.5f);
    float y = clampf(py, 0.5f, (float)ny - 1.5f);
    col = (int)fminf(__fsub_rn(x, 0.5f), (float)(nx - 3));
    row = (int)fminf(__fsub_rn(y, 0.5f), (float)(ny - 3));
}

// A segmented warp sum of `N` amounts per lane, by key (Scatter.segmentedDeposit,
// Scatter.java:385-439): run starts by a max-scan of the lanes that begin a run, Hillis-Steele
// rounds that add only from lanes at or after the run start; returns whether this lane is its
// run's last (and so holds the run's sum).
template <int N>
__device__ __forceinline__ bool segmented_sum(float (&amt)[N], int key) {
    const unsigned all = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    int below = __shfl_up_sync(all, key, 1);
    int head = (lane > 0 && below == key) ? 0 : lane;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int h = __shfl_up_sync(all, head, o);
        if (lane >= o) head = max(head, h);
    }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const bool take = lane - o >= head;
#pragma unroll
        for (int j = 0; j < N; j++) {
            float from = __shfl_up_sync(all, amt[j], o);
            if (take) amt[j] += from;
        }
    }
    int above = __shfl_down_sync(all, key, 1);
    return lane == 31 || above != key;
}

// Flip.scatter's 27 amounts of one particle (Flip.java:269-303) added to acc (the same arithmetic as
// scatter_amounts2, each amount formed and then added).
__device__ __forceinline__ void scatter_accumulate2(const Stencil2& s, float m, float u, float w, float c00, float c01,
                                                    float c10, float c11, float sp, float (&acc)[27]) {
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const float wgt = s.wx[k % 3] * s.wy[k / 3];
        const float wm = wgt * m;
        const float dx = (float)(k % 3) - s.fx, dy = (float)(k / 3) - s.fy;
        const float velU = u + (c00 * dx + c01 * dy);
        const float velV = w + (c10 * dx + c11 * dy);
        acc[3 * k] += wm;
        acc[3 * k + 1] += wm * velU + wgt * (sp * dx);
        acc[3 * k + 2] += wm * velV + wgt * (sp * dy);
    }
}

// Flip.scatter's 27 amounts of one particle (Flip.java:269-303): for stencil node k (k % 3 across,
// k / 3 up), mass w m and the momentum w m (v + C d) + w s d, d = node - f.
__device__ __forceinline__ void scatter_amounts2(const Stencil2& s, float m, float u, float w, float c00, float c01,
                                                 float c10, float c11, float sp, float (&amt)[27]) {
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const float wgt = s.wx[k % 3] * s.wy[k / 3];
        const float wm = wgt * m;
        const float dx = (float)(k % 3) - s.fx, dy = (float)(k / 3) - s.fy;
        const float velU = u + (c00 * dx + c01 * dy);
        const float velV = w + (c10 * dx + c11 * dy);
        amt[3 * k] = wm;
        amt[3 * k + 1] = wm * velU + wgt * (sp * dx);
        amt[3 * k + 2] = wm * velV + wgt * (sp * dy);
    }
}

// Flip.grid (Flip.java:366-412) for one node: momentum over mass plus a step of gravity, zero for
// an empty node; the wall ring drops the velocity into the wall, or a sticky wall stops it.
__device__ __forceinline__ float2 grid_velocity2(float m, float mu, float mv, int ni, int nj, int nx, int ny,
                                                 const Params2& q) {
    float u = 0.0f, w = 0.0f;
    if (m > EMPTY2) {
        u = __fadd_rn(__fdiv_rn(mu, m), __fmul_rn(q.dt, q.gx));
        w = __fadd_rn(__fdiv_rn(mv, m), __fmul_rn(q.dt, q.gy));
    }
    if (q.sticky > 0) {
        const int t = q.sticky;
        if (ni < t || ni > nx - 1 - t || nj < t || nj > ny - 1 - t) u = w = 0.0f;
    } else {
        if (!(ni > 1)) u = fmaxf(u, 0.0f);
        if (ni > nx - 3) u = fminf(u, 0.0f);
        if (!(nj > 1)) w = fmaxf(w, 0.0f);
        if (nj > ny - 3) w = fminf(w, 0.0f);
    }
    return make_float2(u, w);
}

// Flip.keepInside (Flip.java:548-559)
__device__ __forceinline__ void keep_inside2(float& at, float& vel, int size) {
    const float lo = 1.0f, hi = (float)size - 2.0f;
    if (at < lo) {
        at = lo;
        vel = fmaxf(vel, 0.0f);
    }
    if (at > hi) {
        at = hi;
        vel = fminf(vel, 0.0f);
    }
}

// Flip.advectBody (Flip.java:494-545) of one particle, given its stencil and the node velocities
// through vel(k) for stencil node k: the velocity and affine matrix gathered, the position moved
// and kept inside, J updated and clamped. With q.relaxing (Flip.advectRelaxing, Flip.java:451-464, 512-541),
// the stencil's mass density(k) summed too, and J drawn toward rho0 / density at q.relax per second wherever
// that density is at least RELAX_MIN_DENSITY2 of rest.
struct Advected2 {
    float x, y, u, w, c00, c01, c10, c11, j;
};

template <class Vel, class Mass>
__device__ __forceinline__ Advected2 advect2(const Stencil2& s, float px, float py, float pj, int nx, int ny,
                                             const Params2& q, Vel vel, Mass mass) {
    float u = 0, w = 0, b00 = 0, b01 = 0, b10 = 0, b11 = 0, density = 0;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        const float wgt = s.wx[k % 3] * s.wy[k / 3];
        const float dx = (float)(k % 3) - s.fx, dy = (float)(k / 3) - s.fy;
        const float2 g = vel(k);
        const float ui = wgt * g.x, vi = wgt * g.y;
        u += ui;
        w += vi;
        if (q.relaxing) density = __fadd_rn(density, __fmul_rn(wgt, mass(k)));
        b00 += ui * dx;
        b01 += ui * dy;
        b10 += vi * dx;
        b11 += vi * dy;
    }
    Advected2 a;
    a.c00 = 4.0f * b00;
    a.c01 = 4.0f * b01;
    a.c10 = 4.0f * b10;
    a.c11 = 4.0f * b11;
    a.x = px + q.dt * u;
    a.y = py + q.dt * w;
    keep_inside2(a.x, u, nx);
    keep_inside2(a.y, w, ny);
    a.u = u;
    a.w = w;
    float j = pj * (1.0f + q.dt * (a.c00 + a.c11));
    if (q.relaxing && density > __fmul_rn(RELAX_MIN_DENSITY2, q.rho0)) {
        const float measured = __fdiv_rn(q.rho0, density);
        j = __fadd_rn(j, __fmul_rn(__fmul_rn(q.relax, q.dt), __fsub_rn(measured, j)));
    }
    a.j = clampf(j, 1.0f / J_BOUND2, J_BOUND2);
    return a;
}

}  // namespace vf
