// mpm3_kernels.cu -- kernels of the 3D MLS-MPM/APIC step. See mpm3_kernels.cuh for the layout.
// Reference: vexelray-sim-fluid-core/src/main/java/dev/vexelray/sim/fluid/particle/Flip3.java.
#include "mpm3_kernels.cuh"

namespace vf {

// ------------------------------------------------------------------ key + count (standalone)

// The sort's count pass over the current positions, for a step whose previous G2P did not
// count them (the first step after a load or a write of positions).
__global__ void __launch_bounds__(256) k_key_count3(Step3 s) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < s.np;
    int key = 0;
    if (valid) key = key3_of(s.in[X * s.stride + i], s.in[Y * s.stride + i], s.in[Z * s.stride + i], s.d);
    int r = warp_count(s.cell_count, key, valid, s.nkeys, s.status);
    warp_tally(s.brick_count, key >> 9, valid, s.nbricks, s.status);
    if (valid) {
        s.key[i] = key;
        s.rank[i] = r;
    }
}

// ------------------------------------------------------------------ P2G: direct atomics

// One thread per particle: Flip3.scatter (Flip3.java:193-246) in the reference's arithmetic, each
// of the 27 nodes receiving {w m, momentum} in one 16-byte vector reduction.
__global__ void __launch_bounds__(256) k_p2g3_atomic(Step3 s) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= s.np) return;
    const int src = s.perm ? s.perm[d] : d;
    const float* in = s.in;
    const int64_t st = s.stride;
    const float m = in[M * st + src];
    if (!(m > 0.0f)) return;
    const Params3 p = *s.params;
    int cell[3];
    float off[3], w[3][3];
    stencil_axis(in[X * st + src], s.d.nx, cell[0], off[0]);
    stencil_axis(in[Y * st + src], s.d.ny, cell[1], off[1]);
    stencil_axis(in[Z * st + src], s.d.nz, cell[2], off[2]);
#pragma unroll
    for (int a = 0; a < 3; a++) bspline_weights(off[a], w[a]);
    const float vel[3] = {in[U * st + src], in[V * st + src], in[W * st + src]};
    float c[9];
#pragma unroll
    for (int a = 0; a < 9; a++) c[a] = in[(C00 + a) * st + src];
    const float sp = impulse_factor(p.dt, m, p.rho0, p.bulk, in[J * st + src], p.tait);
    const int nx = s.d.nx, ny = s.d.ny;
    const int64_t base = ((int64_t)cell[2] * ny + cell[1]) * nx + cell[0];
#pragma unroll
    for (int k = 0; k < 27; k++) {
        const int ox = k % 3, oy = (k / 3) % 3, oz = k / 9;
        const float wgt = w[0][ox] * (w[1][oy] * w[2][oz]);
        const float dd[3] = {(float)ox - off[0], (float)oy - off[1], (float)oz - off[2]};
        const float wm = wgt * m;
        float mom[3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const float at3 = vel[a] + (c[3 * a] * dd[0] + (c[3 * a + 1] * dd[1] + c[3 * a + 2] * dd[2]));
            mom[a] = wm * at3 + wgt * (sp * dd[a]);
        }
        const int64_t node = base + (int64_t)oz * nx * ny + oy * nx + ox;
        red_add_v4(&s.grid[node], wm, mom[0], mom[1], mom[2]);
    }
}

// ------------------------------------------------------------------ P2G: warp-segmented

// One thread per particle; each run of lanes in one stencil cell is summed across the warp first
// (Scatter.segmentedDeposit, Scatter.java:385-439: run starts by a max-scan, Hillis-Steele within
// runs, the run's last lane takes the atomics), over 27 nodes x 4 fields.
__global__ void __launch_bounds__(256) k_p2g3_warp(Step3 s) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const unsigned all = 0xffffffffu;
    const int64_t st = s.stride;
    const float* in = s.in;
    const int nx = s.d.nx, ny = s.d.ny;
    float amt[27][4];
#pragma unroll
    for (int k = 0; k < 27; k++) amt[k][0] = amt[k][1] = amt[k][2] = amt[k][3] = 0.0f;
    int64_t key = -1;
    if (d < s.np) {
        const int src = s.perm ? s.perm[d] : d;
        const float m = in[M * st + src];
        if (m > 0.0f) {
            const Params3 p = *s.params;
            int cell[3];
            float off[3], w[3][3];
            stencil_axis(in[X * st + src], s.d.nx, cell[0], off[0]);
            stencil_axis(in[Y * st + src], s.d.ny, cell[1], off[1]);
            stencil_axis(in[Z * st + src], s.d.nz, cell[2], off[2]);
#pragma unroll
            for (int a = 0; a < 3; a++) bspline_weights(off[a], w[a]);
            const float vel[3] = {in[U * st + src], in[V * st + src], in[W * st + src]};
            float c[9];
#pragma unroll
            for (int a = 0; a < 9; a++) c[a] = in[(C00 + a) * st + src];
            const float sp = impulse_factor(p.dt, m, p.rho0, p.bulk, in[J * st + src], p.tait);
            key = ((int64_t)cell[2] * ny + cell[1]) * nx + cell[0];
#pragma unroll
            for (int k = 0; k < 27; k++) {
                const int ox = k % 3, oy = (k / 3) % 3, oz = k / 9;
                const float wgt = w[0][ox] * (w[1][oy] * w[2][oz]);
                const float dd[3] = {(float)ox - off[0], (float)oy - off[1], (float)oz - off[2]};
                const float wm = wgt * m;
                amt[k][0] = wm;
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    const float at3 = vel[a] + (c[3 * a] * dd[0] + (c[3 * a + 1] * dd[1] + c[3 * a + 2] * dd[2]));
                    amt[k][1 + a] = wm * at3 + wgt * (sp * dd[a]);
                }
            }
        }
    }
    // Where this lane's run begins: a max-scan over the lanes that start a run.
    const int64_t below = __shfl_up_sync(all, key, 1);
    int head = (lane > 0 && below == key) ? 0 : lane;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int h = __shfl_up_sync(all, head, o);
        if (lane >= o) head = max(head, h);
    }
    const int run_start = head;
    // Hillis-Steele within runs: each shuffle reads every lane's value before any lane adds.
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const bool take = lane - o >= run_start;
#pragma unroll
        for (int k = 0; k < 27; k++) {
#pragma unroll
            for (int f = 0; f < 4; f++) {
                float from = __shfl_up_sync(all, amt[k][f], o);
                if (take) amt[k][f] += from;
            }
        }
    }
    const int64_t above = __shfl_down_sync(all, key, 1);
    const bool last = lane == 31 || above != key;
    if (key >= 0 && last) {
#pragma unroll
        for (int k = 0; k < 27; k++) {
            const int ox = k % 3, oy = (k / 3) % 3, oz = k / 9;
            const int64_t node = key + (int64_t)oz * nx * ny + oy * nx + ox;
            red_add_v4(&s.grid[node], amt[k][0], amt[k][1], amt[k][2], amt[k][3]);
        }
    }
}

// ------------------------------------------------------------------ P2G: sorted brick tile

// One CTA per non-empty 8^3-cell brick (persistent over the list). Each thread owns one stencil
// cell of the brick and sums the 27 x 4 deposits of that cell's particles in registers; the cell
// sums land in a shared-memory window of the brick's 10^3 nodes (no two lanes of a warp hit one
// node, since their cells differ), and the window goes to HBM with one vector reduction per
// touched node. The per-particle arithmetic is Flip3.scatter's, regrouped so each node costs one
// weight, one mass FMA and three momentum FMAs:
//   momentum_a(node o) = w(o) * (A_a + sum_e B_ae o_e),
//   A_a = m (v_a - sum_e C_ae f_e) - s f_a,   B_ae = m C_ae + s [a == e],
// which is (w m)(v_a + C_a . d) + w s d_a with d = o - f.
constexpr int P2G_THREADS = 256;

__global__ void __launch_bounds__(P2G_THREADS) k_p2g3_tile(Step3 s) {
    __shared__ float win[4][WIN3];
    const Params3 p = *s.params;
    const Dims3 dm = s.d;
    const int64_t st = s.stride;
    const float* in = s.in;
    const int na = *s.n_active;
    for (int a = blockIdx.x; a < na; a += gridDim.x) {
        const int b = s.active[a];
        const int bx = b % dm.nbx, by = (b / dm.nbx) % dm.nby, bz = b / (dm.nbx * dm.nby);
        const int cx0 = bx * BRICK, cy0 = by * BRICK, cz0 = bz * BRICK;
        for (int i = threadIdx.x; i < 4 * WIN3; i += P2G_THREADS) (&win[0][0])[i] = 0.0f;
        __syncthreads();
        const int be = s.brick_start[b + 1];
        for (int c = threadIdx.x; c < 512; c += P2G_THREADS) {
            const int64_t key = (int64_t)b * 512 + c;
            int s0 = s.cell_start[key];
            int s1 = c < 511 ? s.cell_start[key + 1] : be;
            if (s0 < 0 || s1 > s.np) {   // a run outside the particles: flagged, and clipped
                set_status(s.status, ST_OOB);
                s0 = max(s0, 0);
                s1 = min(s1, s.np);
            }
            if (s0 >= s1) continue;
            const int lx = c & 7, ly = (c >> 3) & 7, lz = c >> 6;
            float acc[27][4];
#pragma unroll
            for (int k = 0; k < 27; k++) acc[k][0] = acc[k][1] = acc[k][2] = acc[k][3] = 0.0f;
            for (int i = s0; i < s1; i++) {
                const int src = s.perm ? s.perm[i] : i;
                if ((unsigned)src >= (unsigned)s.np) {
                    set_status(s.status, ST_OOB);
                    continue;
                }
                const float m = in[M * st + src];
                if (!(m > 0.0f)) continue;
                int cell[3];
                float f[3];
                stencil_axis(in[X * st + src], dm.nx, cell[0], f[0]);
                stencil_axis(in[Y * st + src], dm.ny, cell[1], f[1]);
                stencil_axis(in[Z * st + src], dm.nz, cell[2], f[2]);
                if (cell[0] != cx0 + lx || cell[1] != cy0 + ly || cell[2] != cz0 + lz) {
                    set_status(s.status, ST_OOB);
                    continue;
                }
                float wx[3], wy[3], wz[3];
                bspline_weights(f[0], wx);
                bspline_weights(f[1], wy);
                bspline_weights(f[2], wz);
                const float sp = impulse_factor(p.dt, m, p.rho0, p.bulk, in[J * st + src], p.tait);
                const float vel[3] = {in[U * st + src], in[V * st + src], in[W * st + src]};
                float A[3], B[3][3];
#pragma unroll
                for (int q = 0; q < 3; q++) {
                    const float c0 = in[(C00 + 3 * q) * st + src], c1 = in[(C00 + 3 * q + 1) * st + src],
                                c2 = in[(C00 + 3 * q + 2) * st + src];
                    const float cf = c0 * f[0] + c1 * f[1] + c2 * f[2];
                    A[q] = m * (vel[q] - cf) - sp * f[q];
                    B[q][0] = m * c0;
                    B[q][1] = m * c1;
                    B[q][2] = m * c2;
                    B[q][q] += sp;
                }
#pragma unroll
                for (int oz = 0; oz < 3; oz++) {
#pragma unroll
                    for (int oy = 0; oy < 3; oy++) {
                        const float wyz = wy[oy] * wz[oz];
                        const float mw = m * wyz;
                        float T[3];
#pragma unroll
                        for (int q = 0; q < 3; q++) T[q] = A[q] + (float)oy * B[q][1] + (float)oz * B[q][2];
#pragma unroll
                        for (int ox = 0; ox < 3; ox++) {
                            const int k = (oz * 3 + oy) * 3 + ox;
                            const float w = wx[ox] * wyz;
                            acc[k][0] += wx[ox] * mw;
#pragma unroll
                            for (int q = 0; q < 3; q++) acc[k][1 + q] += w * (T[q] + (float)ox * B[q][0]);
                        }
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < 27; k++) {
                const int ox = k % 3, oy = (k / 3) % 3, oz = k / 9;
                const int wi = ((lz + oz) * WIN + (ly + oy)) * WIN + (lx + ox);
#pragma unroll
                for (int q = 0; q < 4; q++) atomicAdd(&win[q][wi], acc[k][q]);
            }
        }
        __syncthreads();
        for (int wi = threadIdx.x; wi < WIN3; wi += P2G_THREADS) {
            const float m = win[0][wi];
            if (m == 0.0f && win[1][wi] == 0.0f && win[2][wi] == 0.0f && win[3][wi] == 0.0f) continue;
            const int gx = cx0 + wi % WIN, gy = cy0 + (wi / WIN) % WIN, gz = cz0 + wi / (WIN * WIN);
            if (gx >= dm.nx || gy >= dm.ny || gz >= dm.nz) {
                set_status(s.status, ST_OOB);
                continue;
            }
            red_add_v4(&s.grid[((int64_t)gz * dm.ny + gy) * dm.nx + gx], m, win[1][wi], win[2][wi], win[3][wi]);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ grid update (dense)

__global__ void __launch_bounds__(256) k_grid3_dense(Step3 s) {
    const int64_t nodes = (int64_t)s.d.nx * s.d.ny * s.d.nz;
    const int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= nodes) return;
    const Params3 p = *s.params;
    const int i = (int)(node % s.d.nx), j = (int)((node / s.d.nx) % s.d.ny), k = (int)(node / ((int64_t)s.d.nx * s.d.ny));
    float3 v = grid_velocity(s.grid[node], i, j, k, s.d, p);
    s.vel[node] = make_float4(v.x, v.y, v.z, 0.0f);
}

// ------------------------------------------------------------------ G2P epilogue shared by both forms

// Writes a particle's new state to slot d of the output set and, when the next step sorts,
// counts its new key there.
__device__ __forceinline__ void g2p_store(const Step3& s, int d, const float pos[3], const float vel[3],
                                          const float c[9], float m, float j) {
    float* out = s.out;
    const int64_t st = s.stride;
    out[X * st + d] = pos[0];
    out[Y * st + d] = pos[1];
    out[Z * st + d] = pos[2];
    out[U * st + d] = vel[0];
    out[V * st + d] = vel[1];
    out[W * st + d] = vel[2];
    out[M * st + d] = m;
    out[J * st + d] = j;
#pragma unroll
    for (int a = 0; a < 9; a++) out[(C00 + a) * st + d] = c[a];
}

__device__ __forceinline__ void g2p_count(const Step3& s, int d, bool valid, const float pos[3]) {
    if (!s.count_next) return;
    int key = valid ? key3_of(pos[0], pos[1], pos[2], s.d) : 0;
    int r = warp_count(s.cell_count, key, valid, s.nkeys, s.status);
    warp_tally(s.brick_count, key >> 9, valid, s.nbricks, s.status);
    if (valid) {
        s.key[d] = key;
        s.rank[d] = r;
    }
}

// A particle the reference's advect skips (m <= 0, Flip3.java:342) keeps its state; when the
// step sorts it still moves to its new slot.
__device__ __forceinline__ void g2p_copy(const Step3& s, int d, int src, float pos[3]) {
    const int64_t st = s.stride;
    pos[0] = s.in[X * st + src];
    pos[1] = s.in[Y * st + src];
    pos[2] = s.in[Z * st + src];
    if (s.out != s.in)
        for (int f = 0; f < NF3; f++) s.out[f * st + d] = s.in[f * st + src];
}

// ------------------------------------------------------------------ G2P (dense)

// One thread per particle: Flip3.advect (Flip3.java:329-383) in the reference's arithmetic, over
// the dense velocity grid.
__global__ void __launch_bounds__(256) k_g2p3(Step3 s) {
    const int d = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = d < s.np;
    float pos[3] = {0, 0, 0};
    if (valid) {
        const int src = s.perm ? s.perm[d] : d;
        const int64_t st = s.stride;
        const float m = s.in[M * st + src];
        if (!(m > 0.0f)) {
            g2p_copy(s, d, src, pos);
        } else {
            const Params3 p = *s.params;
            int cell[3];
            float off[3], w[3][3];
            stencil_axis(s.in[X * st + src], s.d.nx, cell[0], off[0]);
            stencil_axis(s.in[Y * st + src], s.d.ny, cell[1], off[1]);
            stencil_axis(s.in[Z * st + src], s.d.nz, cell[2], off[2]);
#pragma unroll
            for (int a = 0; a < 3; a++) bspline_weights(off[a], w[a]);
            const int nx = s.d.nx, ny = s.d.ny;
            const int64_t base = ((int64_t)cell[2] * ny + cell[1]) * nx + cell[0];
            float vel[3] = {0, 0, 0}, sum[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
            for (int k = 0; k < 27; k++) {
                const int ox = k % 3, oy = (k / 3) % 3, oz = k / 9;
                const float wgt = w[0][ox] * (w[1][oy] * w[2][oz]);
                const float dd[3] = {(float)ox - off[0], (float)oy - off[1], (float)oz - off[2]};
                const float4 g = s.vel[base + (int64_t)oz * nx * ny + oy * nx + ox];
                const float gv[3] = {g.x, g.y, g.z};
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    const float na = wgt * gv[a];
                    vel[a] += na;
#pragma unroll
                    for (int e = 0; e < 3; e++) sum[3 * a + e] += na * dd[e];
                }
            }
            float c[9];
#pragma unroll
            for (int a = 0; a < 9; a++) c[a] = 4.0f * sum[a];
            const float at[3] = {s.in[X * st + src], s.in[Y * st + src], s.in[Z * st + src]};
            const int size[3] = {s.d.nx, s.d.ny, s.d.nz};
#pragma unroll
            for (int a = 0; a < 3; a++) {
                pos[a] = at[a] + p.dt * vel[a];
                keep_inside(pos[a], vel[a], size[a]);
            }
            float j = s.in[J * st + src] * (1.0f + p.dt * (c[0] + (c[4] + c[8])));
            j = clampf(j, 1.0f / J_BOUND3, J_BOUND3);
            g2p_store(s, d, pos, vel, c, m, j);
        }
    }
    g2p_count(s, d, valid, pos);
}

// ------------------------------------------------------------------ G2P (brick tile, fused grid update)

// One CTA per non-empty brick. The brick's 10^3 node window is read once from HBM and turned into
// velocities in shared memory (the grid update, Flip3.grid, fused: no velocity grid in HBM), then
// each particle of the brick gathers its 27 nodes from shared memory. The gather is regrouped per
// row of three nodes along x:
//   r0_a = sum_ox wx v_a,  rx_a = wx1 v_a(1) + 2 wx2 v_a(2),
//   vel_a = sum wyz r0_a,  S_ax = sum wyz rx_a,  S_ay = sum oy wyz r0_a,  S_az = sum oz wyz r0_a,
//   C_ae = 4 (S_ae - f_e vel_a)      (= 4 sum w v_a (o_e - f_e), Flip3.java:349-365).
constexpr int G2P_THREADS = 256;

__global__ void __launch_bounds__(G2P_THREADS) k_g2p3_tile(Step3 s) {
    __shared__ float4 vwin[WIN3];
    const Params3 p = *s.params;
    const Dims3 dm = s.d;
    const int64_t st = s.stride;
    const int na = *s.n_active;
    for (int a = blockIdx.x; a < na; a += gridDim.x) {
        const int b = s.active[a];
        const int bx = b % dm.nbx, by = (b / dm.nbx) % dm.nby, bz = b / (dm.nbx * dm.nby);
        const int cx0 = bx * BRICK, cy0 = by * BRICK, cz0 = bz * BRICK;
        for (int wi = threadIdx.x; wi < WIN3; wi += G2P_THREADS) {
            const int gx = cx0 + wi % WIN, gy = cy0 + (wi / WIN) % WIN, gz = cz0 + wi / (WIN * WIN);
            float4 v = make_float4(0, 0, 0, 0);
            if (gx < dm.nx && gy < dm.ny && gz < dm.nz) {
                const float3 u = grid_velocity(s.grid[((int64_t)gz * dm.ny + gy) * dm.nx + gx], gx, gy, gz, dm, p);
                v = make_float4(u.x, u.y, u.z, 0.0f);
            }
            vwin[wi] = v;
        }
        __syncthreads();
        int bs = s.brick_start[b], be = s.brick_start[b + 1];
        if (bs < 0 || be > s.np) {
            set_status(s.status, ST_OOB);
            bs = max(bs, 0);
            be = min(be, s.np);
        }
        // Every thread walks the same number of iterations so the warp-level count is converged.
        const int span = be - bs;
        const int iters = (span + G2P_THREADS - 1) / G2P_THREADS;
        for (int it = 0; it < iters; it++) {
            const int d = bs + it * G2P_THREADS + threadIdx.x;
            const bool valid = d < be;
            float pos[3] = {0, 0, 0};
            if (valid) {
                const int src = s.perm ? s.perm[d] : d;
                const float m = (unsigned)src < (unsigned)s.np ? s.in[M * st + src] : 0.0f;
                if ((unsigned)src >= (unsigned)s.np) {
                    set_status(s.status, ST_OOB);
                } else if (!(m > 0.0f)) {
                    g2p_copy(s, d, src, pos);
                } else {
                    const float at[3] = {s.in[X * st + src], s.in[Y * st + src], s.in[Z * st + src]};
                    int cell[3];
                    float f[3];
                    stencil_axis(at[0], dm.nx, cell[0], f[0]);
                    stencil_axis(at[1], dm.ny, cell[1], f[1]);
                    stencil_axis(at[2], dm.nz, cell[2], f[2]);
                    const int lx = cell[0] - cx0, ly = cell[1] - cy0, lz = cell[2] - cz0;
                    if ((unsigned)lx >= BRICK || (unsigned)ly >= BRICK || (unsigned)lz >= BRICK) {
                        set_status(s.status, ST_OOB);
                        g2p_copy(s, d, src, pos);
                    } else {
                        float wx[3], wy[3], wz[3];
                        bspline_weights(f[0], wx);
                        bspline_weights(f[1], wy);
                        bspline_weights(f[2], wz);
                        const float wx2x2 = 2.0f * wx[2];
                        float vel[3] = {0, 0, 0}, S[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
                        for (int oz = 0; oz < 3; oz++) {
#pragma unroll
                            for (int oy = 0; oy < 3; oy++) {
                                const int w0 = ((lz + oz) * WIN + (ly + oy)) * WIN + lx;
                                const float4 n0 = vwin[w0], n1 = vwin[w0 + 1], n2 = vwin[w0 + 2];
                                const float wyz = wy[oy] * wz[oz];
                                const float v0[3] = {n0.x, n0.y, n0.z}, v1[3] = {n1.x, n1.y, n1.z},
                                            v2[3] = {n2.x, n2.y, n2.z};
#pragma unroll
                                for (int q = 0; q < 3; q++) {
                                    const float r0 = wx[0] * v0[q] + wx[1] * v1[q] + wx[2] * v2[q];
                                    const float rx = wx[1] * v1[q] + wx2x2 * v2[q];
                                    vel[q] += wyz * r0;
                                    S[q][0] += wyz * rx;
                                    if (oy) S[q][1] += ((float)oy * wyz) * r0;
                                    if (oz) S[q][2] += ((float)oz * wyz) * r0;
                                }
                            }
                        }
                        float c[9];
#pragma unroll
                        for (int q = 0; q < 3; q++)
#pragma unroll
                            for (int e = 0; e < 3; e++) c[3 * q + e] = 4.0f * (S[q][e] - f[e] * vel[q]);
                        const int size[3] = {dm.nx, dm.ny, dm.nz};
#pragma unroll
                        for (int q = 0; q < 3; q++) {
                            pos[q] = at[q] + p.dt * vel[q];
                            keep_inside(pos[q], vel[q], size[q]);
                        }
                        float j = s.in[J * st + src] * (1.0f + p.dt * (c[0] + (c[4] + c[8])));
                        j = clampf(j, 1.0f / J_BOUND3, J_BOUND3);
                        g2p_store(s, d, pos, vel, c, m, j);
                    }
                }
            }
            g2p_count(s, d, valid, pos);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ clears and readouts

// Zeroes the node windows of the bricks listed (the bricks a previous scatter into this grid
// buffer touched), so a grid buffer is clean again without a dense memset.
__global__ void __launch_bounds__(256) k_clear_bricks3(Step3 s) {
    const Dims3 dm = s.d;
    const int na = *s.n_active;
    for (int a = blockIdx.x; a < na; a += gridDim.x) {
        const int b = s.active[a];
        const int bx = b % dm.nbx, by = (b / dm.nbx) % dm.nby, bz = b / (dm.nbx * dm.nby);
        const int cx0 = bx * BRICK, cy0 = by * BRICK, cz0 = bz * BRICK;
        for (int wi = threadIdx.x; wi < WIN3; wi += blockDim.x) {
            const int gx = cx0 + wi % WIN, gy = cy0 + (wi / WIN) % WIN, gz = cz0 + wi / (WIN * WIN);
            if (gx < dm.nx && gy < dm.ny && gz < dm.nz)
                s.grid[((int64_t)gz * dm.ny + gy) * dm.nx + gx] = make_float4(0, 0, 0, 0);
        }
    }
}

__global__ void k_touched3(const float4* grid, int64_t nodes, unsigned long long* out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool t = i < nodes && grid[i].x > 0.0f;
    unsigned ballot = __ballot_sync(0xffffffffu, t);
    if ((threadIdx.x & 31) == 0 && ballot) atomicAdd(out, (unsigned long long)__popc(ballot));
}

__global__ void k_unpack_grid3(const float4* grid, float* out, int64_t nodes, int comp) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nodes) return;
    float4 g = grid[i];
    out[i] = comp == 0 ? g.x : comp == 1 ? g.y : comp == 2 ? g.z : g.w;
}

}  // namespace vf
