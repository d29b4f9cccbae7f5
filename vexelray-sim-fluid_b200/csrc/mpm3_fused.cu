// mpm3_fused.cu -- the 3D step's gather and the next step's scatter in one kernel (Flip3.advect, then
// Flip3.scatter of the advected particle: Flip3.java:329-383, 193-246), for sm_100a.
//
// A step of Flip3Step is clear, scatter, grid, advect (Flip3Step.java:81-118). The scatter of step k+1 reads
// exactly the state the advect of step k writes, so the two are fused: the kernel reads a particle's position,
// mass and J once (through the sort's permutation), gathers its new velocity and affine matrix from the grid of
// step k, moves it, writes its new state to its sorted slot, and scatters that new state into the grid of step
// k+1. The 12 velocity and affine floats a particle carries between the two passes never leave registers, so a
// step moves about 100 bytes a particle instead of the separate passes' 170.
//
// Work: one CTA per unit of 8 x 8 x 4 stencil cells of a non-empty brick (two units a brick), persistent.
//   1. the unit's cell starts; each cell's run cut into chunks of up to K consecutive particles;
//   2. the unit's 10 x 10 x 6 node window of grid k turned into node velocities in shared memory (Flip3.grid
//      fused), and a zeroed window of the same nodes for the scatter's sums;
//   3. a thread per chunk: each particle gathered from the velocity window, advected, written out; the chunk's
//      particles still in the chunk's cell sum their 27 nodes' four amounts in registers and add them into the
//      scatter window with one shared-memory reduction per node and amount (K particles' worth at a time);
//      a particle that left its cell (a "mover") adds its own amounts, into the window when its stencil lies
//      inside it, else straight into grid k+1;
//   4. the scatter window's touched nodes added into grid k+1 (one 16-byte vector reduction a node).
// It also counts the next sort's keys: a chunk's particles that stayed add their count to their cell at once.
//
// Windows are laid out 40 floats a (y, z) row, node x and field f at x + 10 f: for the 32 consecutive cells of a
// warp (8 along x, 4 along y) every node offset then maps the lanes to 32 different banks.
#include <climits>

#include "mpm3_kernels.cuh"

namespace vf {

constexpr int FU_THREADS = 256;
constexpr int FU_UZ = 4;                        // unit depth in cells
constexpr int FU_CELLS = BRICK * BRICK * FU_UZ;  // 256: one cell a thread in the unit's scans
constexpr int FU_UNITS_PER_BRICK = BRICK / FU_UZ;
constexpr int FU_WZ = FU_UZ + 2;                // window depth in nodes
constexpr int FU_ROW = 40;                      // floats a (y, z) row: 10 nodes x up to 4 fields
constexpr int FU_PLANE = FU_ROW * WIN;          // 400
constexpr int FU_WIN = FU_PLANE * FU_WZ;        // 2,400 floats a window
constexpr int FU_NODES = WIN * WIN * FU_WZ;     // 600 nodes a window

__device__ __forceinline__ int fu_at(int x, int y, int z) { return x + FU_ROW * y + FU_PLANE * z; }

struct FusedShared {
    float vwin[FU_WIN];          // grid k's node velocities: field f (u, v, w) of node at fu_at + 10 f
    float pwin[FU_WIN];          // grid k+1's sums: field f (m, mu, mv, mw) at fu_at + 10 f
    int cs[FU_CELLS + 1];        // cell c's particles are slots [cs[c], cs[c + 1])
    int off[FU_CELLS + 1];       // cell c's chunks are [off[c], off[c + 1])
    int tmp[FU_THREADS / 32];
    int brick_n;                 // particles of this unit that stayed in their cell
};

// Inclusive scan over the CTA (sum, or running maximum), one value a thread.
template <bool MAX>
__device__ __forceinline__ int fu_scan(int v, int* tmp) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v = MAX ? max(v, y) : v + y;
    }
    if (lane == 31) tmp[warp] = v;
    __syncthreads();
    if (warp == 0) {
        int t = lane < FU_THREADS / 32 ? tmp[lane] : (MAX ? INT_MIN : 0);
#pragma unroll
        for (int o = 1; o < FU_THREADS / 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t = MAX ? max(t, y) : t + y;
        }
        if (lane < FU_THREADS / 32) tmp[lane] = t;
    }
    __syncthreads();
    if (warp > 0) v = MAX ? max(v, tmp[warp - 1]) : v + tmp[warp - 1];
    __syncthreads();
    return v;
}

// One particle's key counted for the next sort (the cell and its brick), outside any warp-wide step.
__device__ __forceinline__ void tally_one(const Step3& s, int key) {
    if ((unsigned)key < (unsigned)s.nkeys) {
        atomicAdd(s.cell_count + key, 1);
        atomicAdd(s.brick_count + (key >> 9), 1);
    } else {
        set_status(s.status, ST_OOB);
    }
}

__device__ __forceinline__ void red_shared(float* addr, float v) {
    asm volatile("red.shared.add.f32 [%0], %1;" ::"r"((unsigned)__cvta_generic_to_shared(addr)), "f"(v) : "memory");
}

// A particle's scatter amounts in the regrouped form the tiled scatter uses: the node at offset o receives
// m w(o) and w(o) (A_a + sum_e B_ae o_e), A_a = m (v_a - C_a . f) - s f_a, B_ae = m C_ae + s [a == e].
struct P2GState {
    float f[3], m, A[3], B[9];
};

__device__ __forceinline__ void p2g_state(P2GState& q, const float f[3], float m, const float vel[3], const float c[9],
                                          float sp) {
#pragma unroll
    for (int e = 0; e < 3; e++) q.f[e] = f[e];
    q.m = m;
#pragma unroll
    for (int r = 0; r < 3; r++) {
        const float c0 = c[3 * r], c1 = c[3 * r + 1], c2 = c[3 * r + 2];
        q.A[r] = m * (vel[r] - (c0 * f[0] + c1 * f[1] + c2 * f[2])) - sp * f[r];
        q.B[3 * r] = m * c0;
        q.B[3 * r + 1] = m * c1;
        q.B[3 * r + 2] = m * c2;
        q.B[3 * r + r] += sp;
    }
}

__device__ __forceinline__ void fu_weights(float f, float w[3]) {
    const float ta = 1.5f - f, tc = f - 1.0f, te = f - 0.5f;
    w[0] = 0.5f * (ta * ta);
    w[1] = 0.75f - tc * tc;
    w[2] = 0.5f * (te * te);
}

// One particle's 27 nodes, each of the four amounts added on its own: into the scatter window at window
// coordinates (wx0, wy0, wz0), or, with win == null, into the grid at node (gx, gy, gz) + offset.
__device__ __forceinline__ void scatter_one(const P2GState& q, float* win, int wx0, int wy0, int wz0, float4* grid,
                                            const Dims3& dm, int gx, int gy, int gz) {
    float wx[3], wy[3], wz[3];
    fu_weights(q.f[0], wx);
    fu_weights(q.f[1], wy);
    fu_weights(q.f[2], wz);
#pragma unroll
    for (int oz = 0; oz < 3; oz++)
#pragma unroll
        for (int oy = 0; oy < 3; oy++)
#pragma unroll
            for (int ox = 0; ox < 3; ox++) {
                const float w = wx[ox] * (wy[oy] * wz[oz]);
                float mom[3];
#pragma unroll
                for (int a = 0; a < 3; a++)
                    mom[a] = w * (q.A[a] + (float)ox * q.B[3 * a] + (float)oy * q.B[3 * a + 1] + (float)oz * q.B[3 * a + 2]);
                if (win) {
                    float* n = win + fu_at(wx0 + ox, wy0 + oy, wz0 + oz);
                    red_shared(n, w * q.m);
                    red_shared(n + 10, mom[0]);
                    red_shared(n + 20, mom[1]);
                    red_shared(n + 30, mom[2]);
                } else {
                    red_add_v4(grid + ((int64_t)(gz + oz) * dm.ny + (gy + oy)) * dm.nx + (gx + ox), w * q.m, mom[0],
                               mom[1], mom[2]);
                }
            }
}

template <int K>
__global__ void __launch_bounds__(FU_THREADS, 2) k_g2p2g3(Step3 s, float4* __restrict__ grid_out) {
    __shared__ FusedShared S;
    const Params3 p = *s.params;
    const Dims3 dm = s.d;
    const int64_t st = s.stride;
    const float* __restrict__ in = s.in;
    float* __restrict__ out = s.out;
    const float4* __restrict__ grid_in = s.grid;
    const int tid = threadIdx.x;
    const float vol = __fdiv_rn(1.0f, p.rho0);   // V0 = m / rho0 as m * (1/rho0)
    const float k4dt = 4.0f * p.dt;
    const int size[3] = {dm.nx, dm.ny, dm.nz};
    const int units = *s.n_active * FU_UNITS_PER_BRICK;
    for (int u = blockIdx.x; u < units; u += gridDim.x) {
        const int b = s.active[u / FU_UNITS_PER_BRICK], lz0 = (u % FU_UNITS_PER_BRICK) * FU_UZ;
        if ((unsigned)b >= (unsigned)s.nbricks) {   // CTA-uniform: every thread read the same entry
            if (tid == 0) set_status(s.status, ST_OOB);
            continue;
        }
        const int bx = b % dm.nbx, by = (b / dm.nbx) % dm.nby, bz = b / (dm.nbx * dm.nby);
        const int cx0 = bx * BRICK, cy0 = by * BRICK, cz0 = bz * BRICK + lz0;
        int bs = s.brick_start[b], be = s.brick_start[b + 1];
        if (bs < 0 || be > s.np || be < bs) {
            if (tid == 0) set_status(s.status, ST_OOB);
            bs = max(bs, 0);
            be = min(max(be, bs), s.np);
        }
        // 1. cell starts, clamped into the brick and made non-decreasing; chunks per cell
        const int64_t key0 = (int64_t)b * 512 + lz0 * 64;
        int v = s.cell_start[key0 + tid];
        int vend = be;   // the unit's end: the next unit's first start, or the brick's end
        if (tid == FU_CELLS - 1 && lz0 + FU_UZ < BRICK) vend = s.cell_start[key0 + FU_CELLS];
        if (v < bs || v > be || vend < bs || vend > be) {
            set_status(s.status, ST_OOB);
            v = min(max(v, bs), be);
            vend = min(max(vend, bs), be);
        }
        v = fu_scan<true>(v, S.tmp);
        S.cs[tid] = v;
        if (tid == FU_CELLS - 1) S.cs[FU_CELLS] = max(v, vend);
        if (tid == 0) S.brick_n = 0;
        __syncthreads();
        const int count = S.cs[tid + 1] - S.cs[tid];
        const int chunks = fu_scan<false>((count + K - 1) / K, S.tmp);
        S.off[tid + 1] = chunks;
        if (tid == 0) S.off[0] = 0;
        // 2. the windows: grid k's velocities (Flip3.grid on the window's nodes), the scatter's zeroed sums
        for (int i = tid; i < FU_NODES; i += FU_THREADS) {
            const int x = i % WIN, y = (i / WIN) % WIN, z = i / (WIN * WIN);
            const int gx = cx0 + x, gy = cy0 + y, gz = cz0 + z;
            float3 vel = make_float3(0.0f, 0.0f, 0.0f);
            if (gx < dm.nx && gy < dm.ny && gz < dm.nz)
                vel = grid_velocity(grid_in[((int64_t)gz * dm.ny + gy) * dm.nx + gx], gx, gy, gz, dm, p);
            float* vn = S.vwin + fu_at(x, y, z);
            vn[0] = vel.x;
            vn[10] = vel.y;
            vn[20] = vel.z;
            float* pn = S.pwin + fu_at(x, y, z);
            pn[0] = pn[10] = pn[20] = pn[30] = 0.0f;
        }
        __syncthreads();
        const int total = S.off[FU_CELLS];
        int stayed = 0;   // this thread's particles that stayed in their cell
        for (int q = tid; q < total; q += FU_THREADS) {
            // 3. the chunk's cell: the last c with off[c] <= q
            int lo = 0, hi = FU_CELLS;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (S.off[mid] <= q) lo = mid;
                else hi = mid;
            }
            const int c = lo;
            const int p0 = S.cs[c] + (q - S.off[c]) * K;
            const int len = min(K, S.cs[c + 1] - p0);
            const int lx = c & 7, ly = (c >> 3) & 7, lz = c >> 6;
            const int gcx = cx0 + lx, gcy = cy0 + ly, gcz = cz0 + lz;   // the cell: the chunk's stencil base
            int src[K];
            float px[K], py[K], pz[K], pm[K], pj[K];
#pragma unroll
            for (int i = 0; i < K; i++) {
                src[i] = -1;
                if (i < len) {
                    int v = s.perm[p0 + i];
                    if ((unsigned)v >= (unsigned)s.np) {
                        set_status(s.status, ST_OOB);
                        v = 0;
                    }
                    src[i] = v;
                    px[i] = in[X * st + v];
                    py[i] = in[Y * st + v];
                    pz[i] = in[Z * st + v];
                    pm[i] = in[M * st + v];
                    pj[i] = in[J * st + v];
                }
            }
            P2GState ps[K];
            bool agg[K];
            int nagg = 0;
#pragma unroll
            for (int i = 0; i < K; i++) {
                agg[i] = false;
                if (i >= len) continue;
                const int d = p0 + i;
                const float at[3] = {px[i], py[i], pz[i]};
                int cl[3];
                float f[3];
                stencil_axis(at[0], dm.nx, cl[0], f[0]);
                stencil_axis(at[1], dm.ny, cl[1], f[1]);
                stencil_axis(at[2], dm.nz, cl[2], f[2]);
                const bool mine = cl[0] == gcx && cl[1] == gcy && cl[2] == gcz;
                if (!(pm[i] > 0.0f) || !mine) {
                    // Flip3.advect skips a particle without mass (Flip3.java:342) and so does the scatter; a
                    // particle outside its sorted cell is a sort fault. Either keeps its state.
                    if (pm[i] > 0.0f) set_status(s.status, ST_OOB);
                    for (int fld = 0; fld < NF3; fld++) out[fld * st + d] = in[fld * st + src[i]];
                    const int key = key3_of(at[0], at[1], at[2], dm);
                    s.key[d] = key;
                    tally_one(s, key);
                    continue;
                }
                // the gather from the velocity window, regrouped per row of three nodes along x
                float wx[3], wy[3], wz[3];
                bspline_weights(f[0], wx);
                bspline_weights(f[1], wy);
                bspline_weights(f[2], wz);
                const float wx2x2 = 2.0f * wx[2];
                float vel[3] = {0, 0, 0}, Sg[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
                for (int oz = 0; oz < 3; oz++) {
#pragma unroll
                    for (int oy = 0; oy < 3; oy++) {
                        const float* r = S.vwin + fu_at(lx, ly + oy, lz + oz);
                        const float wyz = wy[oy] * wz[oz];
#pragma unroll
                        for (int a = 0; a < 3; a++) {
                            const float v0 = r[10 * a], v1 = r[10 * a + 1], v2 = r[10 * a + 2];
                            const float r0 = wx[0] * v0 + wx[1] * v1 + wx[2] * v2;
                            const float rx = wx[1] * v1 + wx2x2 * v2;
                            vel[a] += wyz * r0;
                            Sg[a][0] += wyz * rx;
                            if (oy) Sg[a][1] += ((float)oy * wyz) * r0;
                            if (oz) Sg[a][2] += ((float)oz * wyz) * r0;
                        }
                    }
                }
                float cm[9];
#pragma unroll
                for (int a = 0; a < 3; a++)
#pragma unroll
                    for (int e = 0; e < 3; e++) cm[3 * a + e] = 4.0f * (Sg[a][e] - f[e] * vel[a]);
                float pos[3];
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    pos[a] = at[a] + p.dt * vel[a];
                    keep_inside(pos[a], vel[a], size[a]);
                }
                float jn = pj[i] * (1.0f + p.dt * (cm[0] + (cm[4] + cm[8])));
                jn = clampf(jn, 1.0f / J_BOUND3, J_BOUND3);
                out[X * st + d] = pos[0];
                out[Y * st + d] = pos[1];
                out[Z * st + d] = pos[2];
                out[U * st + d] = vel[0];
                out[V * st + d] = vel[1];
                out[W * st + d] = vel[2];
                out[M * st + d] = pm[i];
                out[J * st + d] = jn;
#pragma unroll
                for (int a = 0; a < 9; a++) out[(C00 + a) * st + d] = cm[a];
                // the next step's scatter of the new state
                int ncl[3];
                float nf[3];
                stencil_axis(pos[0], dm.nx, ncl[0], nf[0]);
                stencil_axis(pos[1], dm.ny, ncl[1], nf[1]);
                stencil_axis(pos[2], dm.nz, ncl[2], nf[2]);
                float jp;
                if (p.tait) {
                    const float rj = __frcp_rn(jn), r2 = rj * rj;
                    jp = p.bulk * ((r2 * r2) * r2 - jn);
                } else {
                    jp = p.bulk * (1.0f - jn);
                }
                const float sp = (k4dt * (pm[i] * vol)) * jp;
                p2g_state(ps[i], nf, pm[i], vel, cm, sp);
                const int key = key3_of_cell(ncl[0], ncl[1], ncl[2], dm);
                s.key[d] = key;
                if (ncl[0] == gcx && ncl[1] == gcy && ncl[2] == gcz) {
                    agg[i] = true;
                    nagg++;
                } else {
                    // a mover: its own amounts, into the window if its stencil lies inside it, else into the grid
                    tally_one(s, key);
                    const int wx0 = ncl[0] - cx0, wy0 = ncl[1] - cy0, wz0 = ncl[2] - cz0;
                    const bool inside = (unsigned)wx0 < BRICK && (unsigned)wy0 < BRICK && (unsigned)wz0 < FU_UZ;
                    scatter_one(ps[i], inside ? S.pwin : nullptr, wx0, wy0, wz0, grid_out, dm, ncl[0], ncl[1], ncl[2]);
                }
            }
            if (nagg > 0) {
                // the chunk's particles that stayed: their 27 nodes' amounts summed here, one reduction a node and
                // amount; (mass, x-momentum) and (y-, z-momentum) in paired fp32
                float w3[K][3][3];   // [particle][axis][offset]
#pragma unroll
                for (int i = 0; i < K; i++)
#pragma unroll
                    for (int e = 0; e < 3; e++) fu_weights(ps[i].f[e], w3[i][e]);
#pragma unroll
                for (int oz = 0; oz < 3; oz++) {
#pragma unroll
                    for (int oy = 0; oy < 3; oy++) {
                        float2 a01[3] = {make_float2(0, 0), make_float2(0, 0), make_float2(0, 0)};
                        float2 a23[3] = {make_float2(0, 0), make_float2(0, 0), make_float2(0, 0)};
#pragma unroll
                        for (int i = 0; i < K; i++) {
                            if (!agg[i]) continue;
                            const P2GState& q = ps[i];
                            const float wyz = w3[i][1][oy] * w3[i][2][oz];
                            const float2 w2 = make_float2(wyz, wyz);
                            float2 t01 = make_float2(q.m, q.A[0]), t23 = make_float2(q.A[1], q.A[2]);
                            if (oy) {
                                const float2 f2 = make_float2((float)oy, (float)oy);
                                t01 = __ffma2_rn(f2, make_float2(0.0f, q.B[1]), t01);
                                t23 = __ffma2_rn(f2, make_float2(q.B[4], q.B[7]), t23);
                            }
                            if (oz) {
                                const float2 f2 = make_float2((float)oz, (float)oz);
                                t01 = __ffma2_rn(f2, make_float2(0.0f, q.B[2]), t01);
                                t23 = __ffma2_rn(f2, make_float2(q.B[5], q.B[8]), t23);
                            }
                            const float2 g01 = __fmul2_rn(w2, t01), g23 = __fmul2_rn(w2, t23);
                            const float2 h01 = __fmul2_rn(w2, make_float2(0.0f, q.B[0]));
                            const float2 h23 = __fmul2_rn(w2, make_float2(q.B[3], q.B[6]));
#pragma unroll
                            for (int ox = 0; ox < 3; ox++) {
                                float2 q01 = g01, q23 = g23;
                                if (ox == 1) {
                                    q01 = __fadd2_rn(q01, h01);
                                    q23 = __fadd2_rn(q23, h23);
                                } else if (ox == 2) {
                                    const float2 two = make_float2(2.0f, 2.0f);
                                    q01 = __ffma2_rn(two, h01, q01);
                                    q23 = __ffma2_rn(two, h23, q23);
                                }
                                const float2 x2 = make_float2(w3[i][0][ox], w3[i][0][ox]);
                                a01[ox] = __ffma2_rn(x2, q01, a01[ox]);
                                a23[ox] = __ffma2_rn(x2, q23, a23[ox]);
                            }
                        }
                        float* r = S.pwin + fu_at(lx, ly + oy, lz + oz);
#pragma unroll
                        for (int ox = 0; ox < 3; ox++) {
                            red_shared(r + ox, a01[ox].x);
                            red_shared(r + ox + 10, a01[ox].y);
                            red_shared(r + ox + 20, a23[ox].x);
                            red_shared(r + ox + 30, a23[ox].y);
                        }
                    }
                }
                atomicAdd(s.cell_count + key0 + c, nagg);
                stayed += nagg;
            }
        }
        // the unit's particles that stayed all count toward brick b
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) stayed += __shfl_xor_sync(0xffffffffu, stayed, o);
        if ((tid & 31) == 0 && stayed) atomicAdd(&S.brick_n, stayed);
        __syncthreads();
        if (tid == 0 && S.brick_n) atomicAdd(s.brick_count + b, S.brick_n);
        // 4. the scatter window's touched nodes into grid k+1
        for (int i = tid; i < FU_NODES; i += FU_THREADS) {
            const int x = i % WIN, y = (i / WIN) % WIN, z = i / (WIN * WIN);
            const float* pn = S.pwin + fu_at(x, y, z);
            const float m = pn[0], mu = pn[10], mv = pn[20], mw = pn[30];
            if (m == 0.0f && mu == 0.0f && mv == 0.0f && mw == 0.0f) continue;
            const int gx = cx0 + x, gy = cy0 + y, gz = cz0 + z;
            if (gx >= dm.nx || gy >= dm.ny || gz >= dm.nz) {
                set_status(s.status, ST_OOB);
                continue;
            }
            red_add_v4(grid_out + ((int64_t)gz * dm.ny + gy) * dm.nx + gx, m, mu, mv, mw);
        }
        __syncthreads();
    }
}

#ifndef VF_FUSED_CHUNK
#define VF_FUSED_CHUNK 4
#endif
constexpr int FU_K = VF_FUSED_CHUNK;   // particles a chunk (a build may choose another)

cudaError_t launch_g2p2g3(int blocks, const Step3& s, float4* grid_out, cudaStream_t stream) {
    k_g2p2g3<FU_K><<<blocks, FU_THREADS, 0, stream>>>(s, grid_out);
    return cudaGetLastError();
}

}  // namespace vf
