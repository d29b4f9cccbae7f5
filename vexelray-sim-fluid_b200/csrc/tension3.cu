// tension3.cu -- surface tension for the 3D step (Tension3.java): the colour, its blurs, the capillary stress and
// the grid update with the stress's force; node (k*ny + j)*nx + i. The blurs work on shared-memory tiles, the
// stress and the grid update one thread per node.
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

// Blur tiles: a CTA of 32 x 8 threads blurs 32 x 8 x 8 nodes. It first stages the tile's nodes and a one-node
// halo, each read at its held coordinates, in shared memory (34 x 10 x 10 floats), so every neighbour read of
// the reference is one shared-memory load. For the first blur a staged value is already the node's mass over a
// full node's, no more than one: that depends on the node read alone, so it is formed once per staged node.
constexpr int BT_X = 32, BT_Y = 8, BT_Z = 8;
constexpr int BH_X = BT_X + 2, BH_Y = BT_Y + 2, BH_Z = BT_Z + 2;

}  // namespace

// Tension3.blur (Tension3.java:73-107): the [1 2 1]^3/64 blur of the node mass taken to a colour (SCALED, the
// first blur: src is the grid, float4 {m, ...}) or of the last colour, dk outermost and di innermost, each read
// held to the wall ring; a full node on the wall ring holds half a rest mass for each wall through it.
// Stages the CTA's tile and its halo, each node read at its held coordinates (and for SCALED taken to a colour).
template <bool SCALED>
__device__ __forceinline__ void stage_tile(float (&tile)[BH_Z][BH_Y][BH_X], const void* src, const Params3* params,
                                           const Dims3& d, int x0, int y0, int z0) {
    const int size[3] = {d.nx, d.ny, d.nz};
    const float rho0 = SCALED ? params->rho0 : 0.0f;
    for (int t = threadIdx.y * BT_X + threadIdx.x; t < BH_X * BH_Y * BH_Z; t += BT_X * BT_Y) {
        const int lx = t % BH_X, ly = (t / BH_X) % BH_Y, lz = t / (BH_X * BH_Y);
        const int c[3] = {held(x0 + lx - 1, d.nx), held(y0 + ly - 1, d.ny), held(z0 + lz - 1, d.nz)};
        const int64_t n = index3(d, c[0], c[1], c[2]);
        float value;
        if (SCALED) {
            value = static_cast<const float4*>(src)[n].x;
            float full = rho0;
#pragma unroll
            for (int a = 0; a < 3; a++) {
                if (c[a] == WALL3) full = __fmul_rn(0.5f, full);
                if (c[a] == size[a] - 1 - WALL3) full = __fmul_rn(0.5f, full);
            }
            value = fminf(__fdiv_rn(value, full), 1.0f);
        } else {
            value = static_cast<const float*>(src)[n];
        }
        tile[lz][ly][lx] = value;
    }
    __syncthreads();
}

template <bool SCALED>
__global__ void __launch_bounds__(BT_X * BT_Y) k_tension3_blur_tile(const void* src, float* dst,
                                                                     const Params3* params, Dims3 d) {
    __shared__ float tile[BH_Z][BH_Y][BH_X];
    const int x0 = blockIdx.x * BT_X, y0 = blockIdx.y * BT_Y, z0 = blockIdx.z * BT_Z;
    stage_tile<SCALED>(tile, src, params, d, x0, y0, z0);
    const int i = x0 + threadIdx.x, j = y0 + threadIdx.y;
    if (i >= d.nx || j >= d.ny) return;
    // the 3 x 3 neighbourhood of this (i, j) in three consecutive planes, sliding one plane per output node
    float win[3][9];
#pragma unroll
    for (int p = 0; p < 2; p++)
#pragma unroll
        for (int q = 0; q < 9; q++) win[p + 1][q] = tile[p][threadIdx.y + q / 3][threadIdx.x + q % 3];
#pragma unroll
    for (int tz = 0; tz < BT_Z; tz++) {
#pragma unroll
        for (int q = 0; q < 9; q++) {
            win[0][q] = win[1][q];
            win[1][q] = win[2][q];
            win[2][q] = tile[tz + 2][threadIdx.y + q / 3][threadIdx.x + q % 3];
        }
        const int k = z0 + tz;
        if (k >= d.nz) break;
        float sum = 0.0f;
#pragma unroll
        for (int dk = -1; dk <= 1; dk++) {
#pragma unroll
            for (int dj = -1; dj <= 1; dj++) {
#pragma unroll
                for (int di = -1; di <= 1; di++) {
                    const float weight = (float)((2 - abs(di)) * (2 - abs(dj)) * (2 - abs(dk))) / 64.0f;
                    sum = __fadd_rn(sum, __fmul_rn(weight, win[dk + 1][(dj + 1) * 3 + di + 1]));
                }
            }
        }
        dst[index3(d, i, j, k)] = sum;
    }
}

cudaError_t launch_tension3_blur(bool scaled, const void* src, float* dst, const Params3* params, const Dims3& d,
                                 cudaStream_t stream) {
    const dim3 grid((d.nx + BT_X - 1) / BT_X, (d.ny + BT_Y - 1) / BT_Y, (d.nz + BT_Z - 1) / BT_Z);
    if (scaled)
        k_tension3_blur_tile<true><<<grid, dim3(BT_X, BT_Y), 0, stream>>>(src, dst, params, d);
    else
        k_tension3_blur_tile<false><<<grid, dim3(BT_X, BT_Y), 0, stream>>>(src, dst, params, d);
    return cudaGetLastError();
}

// Tension3.stress (Tension3.java:128-154): the stress over sigma from the colour's central differences g,
// diagonal (|g|^2 - g_a^2)/|g| and off the diagonal -g_a g_b/|g|, |g| kept off zero by EPS. The colour is staged
// as the blurs stage it, so each held neighbour read is a shared-memory load.
__global__ void __launch_bounds__(BT_X * BT_Y) k_tension3_stress(const float* colour, float* stress, Dims3 d) {
    __shared__ float tile[BH_Z][BH_Y][BH_X];
    const int x0 = blockIdx.x * BT_X, y0 = blockIdx.y * BT_Y, z0 = blockIdx.z * BT_Z;
    stage_tile<false>(tile, colour, nullptr, d, x0, y0, z0);
    const int i = x0 + threadIdx.x, j = y0 + threadIdx.y;
    if (i >= d.nx || j >= d.ny) return;
    const int tx = threadIdx.x + 1, ty = threadIdx.y + 1;
    const int64_t n = (int64_t)d.nx * d.ny * d.nz;
    for (int tz = 1; tz <= BT_Z; tz++) {
        const int k = z0 + tz - 1;
        if (k >= d.nz) break;
        float g[3];
        g[0] = __fmul_rn(0.5f, __fsub_rn(tile[tz][ty][tx + 1], tile[tz][ty][tx - 1]));
        g[1] = __fmul_rn(0.5f, __fsub_rn(tile[tz][ty + 1][tx], tile[tz][ty - 1][tx]));
        g[2] = __fmul_rn(0.5f, __fsub_rn(tile[tz + 1][ty][tx], tile[tz - 1][ty][tx]));
        const float xx = __fmul_rn(g[0], g[0]), yy = __fmul_rn(g[1], g[1]), zz = __fmul_rn(g[2], g[2]);
        const float length = __fsqrt_rn(__fadd_rn(__fadd_rn(xx, __fadd_rn(yy, zz)), EPS2));
        const int64_t node = index3(d, i, j, k);
        stress[0 * n + node] = __fdiv_rn(__fadd_rn(yy, zz), length);
        stress[1 * n + node] = __fdiv_rn(__fadd_rn(xx, zz), length);
        stress[2 * n + node] = __fdiv_rn(__fadd_rn(xx, yy), length);
        stress[3 * n + node] = -__fdiv_rn(__fmul_rn(g[0], g[1]), length);
        stress[4 * n + node] = -__fdiv_rn(__fmul_rn(g[0], g[2]), length);
        stress[5 * n + node] = -__fdiv_rn(__fmul_rn(g[1], g[2]), length);
    }
}

cudaError_t launch_tension3_stress(const float* colour, float* stress, const Dims3& d, cudaStream_t stream) {
    const dim3 grid((d.nx + BT_X - 1) / BT_X, (d.ny + BT_Y - 1) / BT_Y, (d.nz + BT_Z - 1) / BT_Z);
    k_tension3_stress<<<grid, dim3(BT_X, BT_Y), 0, stream>>>(colour, stress, d);
    return cudaGetLastError();
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
