// tension3.cu -- surface tension for the 3D step (Tension3.java): the colour, its blurs, the capillary stress and
// the grid update with the stress's force, one thread per node, node (k*ny + j)*nx + i.
//
// Every operation is the reference's, in its order, rounded once (the _rn intrinsics keep the compiler from
// fusing a multiply into an add), so the passes give the same bits as the float restatement on the CPU. Reads of
// a neighbour are held to the wall ring [1, n-2] on every axis, as Tension3.at does (Tension3.java:215-221).
#include "mpm3_kernels.cuh"

namespace vf {

namespace {

constexpr float MIN_COLOUR = 0.3f;    // Tension.MIN_COLOUR (Tension.java:74)
constexpr float MASS_FLOOR = 0.3f;    // Tension.MASS_FLOOR (Tension.java:77)
constexpr float EPS2 = (float)(1e-4 * 1e-4);   // Tension3.EPS squared, formed in double (Tension3.java:57, 145)
constexpr int WALL3 = 1;              // Flip3.WALL

__device__ __forceinline__ int held(int c, int size) { return min(max(c, WALL3), size - 1 - WALL3); }

__device__ __forceinline__ bool node_of(const Dims3& d, int64_t& node, int& i, int& j, int& k) {
    const int64_t nodes = (int64_t)d.nx * d.ny * d.nz;
    node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= nodes) return false;
    i = (int)(node % d.nx);
    j = (int)((node / d.nx) % d.ny);
    k = (int)(node / ((int64_t)d.nx * d.ny));
    return true;
}

__device__ __forceinline__ int64_t index3(const Dims3& d, int i, int j, int k) {
    return ((int64_t)k * d.ny + j) * d.nx + i;
}

// The 27-point [1 2 1]^3/64 blur at (i, j, k), dk outermost and di innermost (Tension3.java:78-104). SCALED: each
// read is the node mass over a full node's, no more than one; a full node on the wall ring holds half a rest mass
// for each wall through it (Tension3.java:84-99).
template <bool SCALED, class Read>
__device__ __forceinline__ float blur_at(const Dims3& d, int i, int j, int k, float rho0, Read read) {
    float sum = 0.0f;
#pragma unroll
    for (int dk = -1; dk <= 1; dk++) {
#pragma unroll
        for (int dj = -1; dj <= 1; dj++) {
#pragma unroll
            for (int di = -1; di <= 1; di++) {
                const float weight = (float)((2 - abs(di)) * (2 - abs(dj)) * (2 - abs(dk))) / 64.0f;
                const int c[3] = {held(i + di, d.nx), held(j + dj, d.ny), held(k + dk, d.nz)};
                float value = read(index3(d, c[0], c[1], c[2]));
                if (SCALED) {
                    const int size[3] = {d.nx, d.ny, d.nz};
                    float full = rho0;
#pragma unroll
                    for (int a = 0; a < 3; a++) {
                        if (c[a] == WALL3) full = __fmul_rn(0.5f, full);
                        if (c[a] == size[a] - 1 - WALL3) full = __fmul_rn(0.5f, full);
                    }
                    value = fminf(__fdiv_rn(value, full), 1.0f);
                }
                sum = __fadd_rn(sum, __fmul_rn(weight, value));
            }
        }
    }
    return sum;
}

}  // namespace

// Tension3.blur(scaled = true): the first blur, of the scatter's node mass (Tension3.java:73-107).
__global__ void __launch_bounds__(256) k_tension3_colour(const float4* grid, float* colour, const Params3* params,
                                                         Dims3 d) {
    int64_t node;
    int i, j, k;
    if (!node_of(d, node, i, j, k)) return;
    const float rho0 = params->rho0;
    colour[node] = blur_at<true>(d, i, j, k, rho0, [&](int64_t n) { return grid[n].x; });
}

// Tension3.blur(scaled = false): a later blur of the colour.
__global__ void __launch_bounds__(256) k_tension3_blur(const float* src, float* dst, Dims3 d) {
    int64_t node;
    int i, j, k;
    if (!node_of(d, node, i, j, k)) return;
    dst[node] = blur_at<false>(d, i, j, k, 0.0f, [&](int64_t n) { return src[n]; });
}

// Tension3.stress (Tension3.java:128-154): the stress over sigma from the colour's central differences g,
// diagonal (|g|^2 - g_a^2)/|g| and off the diagonal -g_a g_b/|g|, |g| kept off zero by EPS.
__global__ void __launch_bounds__(256) k_tension3_stress(const float* colour, float* stress, Dims3 d) {
    int64_t node;
    int i, j, k;
    if (!node_of(d, node, i, j, k)) return;
    const int hi = held(i, d.nx), hj = held(j, d.ny), hk = held(k, d.nz);
    float g[3];
    g[0] = __fmul_rn(0.5f, __fsub_rn(colour[index3(d, held(i + 1, d.nx), hj, hk)],
                                     colour[index3(d, held(i - 1, d.nx), hj, hk)]));
    g[1] = __fmul_rn(0.5f, __fsub_rn(colour[index3(d, hi, held(j + 1, d.ny), hk)],
                                     colour[index3(d, hi, held(j - 1, d.ny), hk)]));
    g[2] = __fmul_rn(0.5f, __fsub_rn(colour[index3(d, hi, hj, held(k + 1, d.nz))],
                                     colour[index3(d, hi, hj, held(k - 1, d.nz))]));
    const float xx = __fmul_rn(g[0], g[0]), yy = __fmul_rn(g[1], g[1]), zz = __fmul_rn(g[2], g[2]);
    const float length = __fsqrt_rn(__fadd_rn(__fadd_rn(xx, __fadd_rn(yy, zz)), EPS2));
    const int64_t n = (int64_t)d.nx * d.ny * d.nz;
    stress[0 * n + node] = __fdiv_rn(__fadd_rn(yy, zz), length);
    stress[1 * n + node] = __fdiv_rn(__fadd_rn(xx, zz), length);
    stress[2 * n + node] = __fdiv_rn(__fadd_rn(xx, yy), length);
    stress[3 * n + node] = -__fdiv_rn(__fmul_rn(g[0], g[1]), length);
    stress[4 * n + node] = -__fdiv_rn(__fmul_rn(g[0], g[2]), length);
    stress[5 * n + node] = -__fdiv_rn(__fmul_rn(g[1], g[2]), length);
}

// Flip3.gridWithTension (Flip3.java:267-310) with Tension3.force (Tension3.java:162-200): the force over sigma on
// a node is the flux of the stress across its six faces, the mean of T_ab at the two nodes a face joins, over
// the faces whose nodes both hold MIN_COLOUR, on nodes of the wall ring or inside it; across a face in the wall
// only the normal stress crosses.
__global__ void __launch_bounds__(256) k_grid3_tension(Step3 s, const float* colour, const float* stress) {
    int64_t node;
    int i, j, k;
    if (!node_of(s.d, node, i, j, k)) return;
    const Dims3 d = s.d;
    const Params3 p = *s.params;
    const float4 g4 = s.grid[node];
    float v[3];
    grid_velocity_free(g4, p, v);
    const float mass = g4.x;
    if (mass > EMPTY3) {
        const int64_t n = (int64_t)d.nx * d.ny * d.nz;
        const int at[3] = {i, j, k};
        const int size[3] = {d.nx, d.ny, d.nz};
        // the stress planes a face along axis a carries, component c: T_ac (txx tyy tzz txy txz tyz)
        const int tensor[3][3] = {{0, 3, 4}, {3, 1, 5}, {4, 5, 2}};
        bool ring = colour[node] > MIN_COLOUR;
#pragma unroll
        for (int a = 0; a < 3; a++) ring = ring && !(at[a] < WALL3) && !(at[a] > size[a] - 1 - WALL3);
        float force[3] = {0.0f, 0.0f, 0.0f};
        if (ring) {
#pragma unroll
            for (int a = 0; a < 3; a++) {
#pragma unroll
                for (int sign = -1; sign <= 1; sign += 2) {
                    int c3[3] = {held(i, d.nx), held(j, d.ny), held(k, d.nz)};
                    c3[a] = held(at[a] + sign, size[a]);
                    const int64_t there = index3(d, c3[0], c3[1], c3[2]);
                    if (!(colour[there] > MIN_COLOUR)) continue;
                    const bool wall = sign < 0 ? !(at[a] > WALL3) : !(at[a] < size[a] - 1 - WALL3);
                    const float shear = wall ? 0.0f : 1.0f;
                    const float half = 0.5f * (float)sign;
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        const float* t = stress + (int64_t)tensor[a][c] * n;
                        const float flux = __fmul_rn(half, __fadd_rn(t[node], t[there]));
                        force[c] = __fadd_rn(force[c], c == a ? flux : __fmul_rn(shear, flux));
                    }
                }
            }
        }
        const float push = __fdiv_rn(__fmul_rn(p.dt, p.sigma), fmaxf(mass, __fmul_rn(MASS_FLOOR, p.rho0)));
#pragma unroll
        for (int a = 0; a < 3; a++) v[a] = __fadd_rn(v[a], __fmul_rn(push, force[a]));
    }
    const float3 w = grid_walls(v, i, j, k, d, p);
    s.vel[node] = make_float4(w.x, w.y, w.z, 0.0f);
}

}  // namespace vf
