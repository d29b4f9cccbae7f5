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

// Windows: float4 per node, node (x, y, z) of the unit's 10 x 10 x (UZ + 2) window at x + 10 y + 100 z.
template <int UZ>
struct FusedUnit {
    static constexpr int T = 64 * UZ;          // threads: one per cell of the unit in its scans
    static constexpr int NW = T / 32;          // warps, each with its own scatter window
    static constexpr int CELLS = 64 * UZ;      // 8 x 8 x UZ stencil cells
    static constexpr int PER_BRICK = BRICK / UZ;
    static constexpr int WN = WIN * WIN * (UZ + 2);   // window nodes
    static constexpr int CAP = 16 * T;         // chunk list entries held at once (rounds beyond are a second batch)
    static constexpr size_t SMEM = sizeof(float4) * (size_t)WN * (1 + NW) + sizeof(int) * (CELLS + 1 + CAP + NW + 4);
};

__device__ __forceinline__ int fu_node(int x, int y, int z) { return x + WIN * y + WIN * WIN * z; }

// Inclusive scan over the CTA (sum, or running maximum), one value a thread; *total gets the CTA's total (sum) or
// maximum, read before the last barrier so the next scan may reuse tmp.
template <int NW, bool MAX>
__device__ __forceinline__ int fu_scan(int v, int* tmp, int* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v = MAX ? max(v, y) : v + y;
    }
    if (lane == 31) tmp[warp] = v;
    __syncthreads();
    if (warp == 0) {
        int t = lane < NW ? tmp[lane] : (MAX ? INT_MIN : 0);
#pragma unroll
        for (int o = 1; o < NW; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t = MAX ? max(t, y) : t + y;
        }
        if (lane < NW) tmp[lane] = t;
    }
    __syncthreads();
    if (warp > 0) v = MAX ? max(v, tmp[warp - 1]) : v + tmp[warp - 1];
    *total = tmp[NW - 1];
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

__device__ __forceinline__ void fu_weights(float f, float w[3]) {
    const float ta = 1.5f - f, tc = f - 1.0f, te = f - 0.5f;
    w[0] = 0.5f * (ta * ta);
    w[1] = 0.75f - tc * tc;
    w[2] = 0.5f * (te * te);
}

// A particle's scatter amounts in the regrouped form the tiled scatter uses: the node at offset o receives
// m w(o) and w(o) (A_a + sum_e B_ae o_e), A_a = m (v_a - C_a . f) - s f_a, B_ae = m C_ae + s [a == e].
struct P2GState {
    float m, A[3], B[9];
    float w[3][3];   // the stencil weights, [axis][offset]
};

__device__ __forceinline__ void p2g_state(P2GState& q, const float f[3], float m, const float vel[3], const float c[9],
                                          float sp) {
#pragma unroll
    for (int e = 0; e < 3; e++) fu_weights(f[e], q.w[e]);
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

// One particle's 27 nodes added into the grid at node (gx, gy, gz) + offset, one 16-byte vector reduction a node
// (a particle that left its sorted cell).
__device__ __forceinline__ void scatter_one(const P2GState& q, float4* grid, const Dims3& dm, int gx, int gy, int gz) {
    const float* wx = q.w[0];
    const float* wy = q.w[1];
    const float* wz = q.w[2];
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
                red_add_v4(grid + ((int64_t)(gz + oz) * dm.ny + (gy + oy)) * dm.nx + (gx + ox), w * q.m, mom[0],
                           mom[1], mom[2]);
            }
}


template <int UZ, int K>
__global__ void __launch_bounds__(FusedUnit<UZ>::T, (UZ == 4 ? 2 : 4)) k_g2p2g3(Step3 s, float4* __restrict__ grid_out) {
    using Unit = FusedUnit<UZ>;
    constexpr int T = Unit::T, NW = Unit::NW, CELLS = Unit::CELLS, WN = Unit::WN, CAP = Unit::CAP;
    extern __shared__ __align__(16) float4 fu_smem[];
    float4* vwin = fu_smem;                                   // grid k's node velocities (u, v, w, 0)
    float4* pwin_all = vwin + WN;                             // NW scatter windows (m, mu, mv, mw)
    int* cs = reinterpret_cast<int*>(pwin_all + NW * WN);     // cell c's slots: [cs[c], cs[c + 1])
    int* list = cs + CELLS + 1;                               // the chunks, round by round: cell | round << 16
    int* tmp = list + CAP;
    int* brick_n = tmp + NW;                                  // particles of the unit that stayed in their cell
    const Params3 p = *s.params;
    const Dims3 dm = s.d;
    const int64_t st = s.stride;
    const float* __restrict__ in = s.in;
    float* __restrict__ out = s.out;
    const float4* __restrict__ grid_in = s.grid;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float4* pwin = pwin_all + warp * WN;
    const float vol = __fdiv_rn(1.0f, p.rho0);   // V0 = m / rho0 as m * (1/rho0)
    const float k4dt = 4.0f * p.dt;
    const int size[3] = {dm.nx, dm.ny, dm.nz};
    const int units = *s.n_active * Unit::PER_BRICK;
    for (int u = blockIdx.x; u < units; u += gridDim.x) {
        const int b = s.active[u / Unit::PER_BRICK], lz0 = (u % Unit::PER_BRICK) * UZ;
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
        if (tid == CELLS - 1 && lz0 + UZ < BRICK) vend = s.cell_start[key0 + CELLS];
        if (v < bs || v > be || vend < bs || vend > be) {
            set_status(s.status, ST_OOB);
            v = min(max(v, bs), be);
            vend = min(max(vend, bs), be);
        }
        int dummy;
        v = fu_scan<NW, true>(v, tmp, &dummy);
        cs[tid] = v;
        if (tid == CELLS - 1) cs[CELLS] = max(v, vend);
        if (tid == 0) *brick_n = 0;
        __syncthreads();
        if (cs[CELLS] == cs[0]) continue;   // an empty unit (CTA-uniform)
        const int nch = (cs[tid + 1] - cs[tid] + K - 1) / K;
        int rounds;
        fu_scan<NW, true>(nch, tmp, &rounds);
        // 2. the windows: grid k's velocities (Flip3.grid on the window's nodes); every warp's scatter window zeroed
        for (int i = tid; i < WN; i += T) {
            const int x = i % WIN, y = (i / WIN) % WIN, z = i / (WIN * WIN);
            const int gx = cx0 + x, gy = cy0 + y, gz = cz0 + z;
            float3 vel = make_float3(0.0f, 0.0f, 0.0f);
            if (gx < dm.nx && gy < dm.ny && gz < dm.nz)
                vel = grid_velocity(grid_in[((int64_t)gz * dm.ny + gy) * dm.nx + gx], gx, gy, gz, dm, p);
            vwin[i] = make_float4(vel.x, vel.y, vel.z, 0.0f);
        }
        for (int i = tid; i < NW * WN; i += T) pwin_all[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        int stayed = 0;   // this thread's particles that stayed in their cell
        // 3. the chunks, round by round: round r holds chunk r of every cell that has one, so the 32 chunks a warp
        // takes at once (rounds padded to whole warps) belong to 32 different cells, and at one stencil offset the
        // lanes add into 32 different nodes of the warp's own window: plain loads and stores, no atomics
        for (int r0 = 0; r0 < rounds;) {
            int filled = 0, r = r0;
            while (r < rounds) {
                const int flag = nch > r ? 1 : 0;
                int cnt;
                const int at = fu_scan<NW, false>(flag, tmp, &cnt) - flag;
                const int padded = (cnt + 31) & ~31;
                if (filled + padded > CAP) break;   // CTA-uniform; a round always fits an empty list
                if (flag) list[filled + at] = tid | (r << 16);
                if (tid < padded - cnt) list[filled + cnt + tid] = -1;
                filled += padded;
                r++;
            }
            __syncthreads();
            for (int pass = warp; pass < filled / 32; pass += NW) {
                const int entry = list[pass * 32 + lane];
                const int c = entry >= 0 ? (entry & 0xffff) : 0;
                const int p0 = entry >= 0 ? cs[c] + (entry >> 16) * K : 0;
                const int len = entry >= 0 ? min(K, cs[c + 1] - p0) : 0;
                const int lx = c & 7, ly = (c >> 3) & 7, lz = c >> 6;
                const int gcx = cx0 + lx, gcy = cy0 + ly, gcz = cz0 + lz;   // the cell: the chunk's stencil base
                int src[K];
                float px[K], py[K], pz[K], pm[K], pj[K];
#pragma unroll
                for (int i = 0; i < K; i++) {
                    src[i] = -1;
                    if (i < len) {
                        int sv = s.perm[p0 + i];
                        if ((unsigned)sv >= (unsigned)s.np) {
                            set_status(s.status, ST_OOB);
                            sv = 0;
                        }
                        src[i] = sv;
                        px[i] = in[X * st + sv];
                        py[i] = in[Y * st + sv];
                        pz[i] = in[Z * st + sv];
                        pm[i] = in[M * st + sv];
                        pj[i] = in[J * st + sv];
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
                    const float at3[3] = {px[i], py[i], pz[i]};
                    int cl[3];
                    float f[3];
                    stencil_axis(at3[0], dm.nx, cl[0], f[0]);
                    stencil_axis(at3[1], dm.ny, cl[1], f[1]);
                    stencil_axis(at3[2], dm.nz, cl[2], f[2]);
                    const bool mine = cl[0] == gcx && cl[1] == gcy && cl[2] == gcz;
                    if (!(pm[i] > 0.0f) || !mine) {
                        // Flip3.advect skips a particle without mass (Flip3.java:342) and so does the scatter; a
                        // particle outside its sorted cell is a sort fault. Either keeps its state.
                        if (pm[i] > 0.0f) set_status(s.status, ST_OOB);
                        for (int fld = 0; fld < NF3; fld++) out[fld * st + d] = in[fld * st + src[i]];
                        const int key = key3_of(at3[0], at3[1], at3[2], dm);
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
                            const int w0 = fu_node(lx, ly + oy, lz + oz);
                            const float4 n0 = vwin[w0], n1 = vwin[w0 + 1], n2 = vwin[w0 + 2];
                            const float wyz = wy[oy] * wz[oz];
                            const float v0[3] = {n0.x, n0.y, n0.z}, v1[3] = {n1.x, n1.y, n1.z},
                                        v2[3] = {n2.x, n2.y, n2.z};
#pragma unroll
                            for (int a = 0; a < 3; a++) {
                                const float r0v = wx[0] * v0[a] + wx[1] * v1[a] + wx[2] * v2[a];
                                const float rx = wx[1] * v1[a] + wx2x2 * v2[a];
                                vel[a] += wyz * r0v;
                                Sg[a][0] += wyz * rx;
                                if (oy) Sg[a][1] += ((float)oy * wyz) * r0v;
                                if (oz) Sg[a][2] += ((float)oz * wyz) * r0v;
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
                        pos[a] = at3[a] + p.dt * vel[a];
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
                        // a mover: its own amounts straight into grid k+1
                        tally_one(s, key);
                        scatter_one(ps[i], grid_out, dm, ncl[0], ncl[1], ncl[2]);
                    }
                }
                // the chunk's particles that stayed: their 27 nodes' amounts summed here ((mass, x-momentum) and
                // (y-, z-momentum) in paired fp32), then added into the warp's window, a row of three nodes at a
                // time with every lane of the warp on the same row
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
                            const float wyz = q.w[1][oy] * q.w[2][oz];
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
                                const float2 x2 = make_float2(q.w[0][ox], q.w[0][ox]);
                                a01[ox] = __ffma2_rn(x2, q01, a01[ox]);
                                a23[ox] = __ffma2_rn(x2, q23, a23[ox]);
                            }
                        }
                        // one node at a time, every lane of the warp on the same node offset between barriers: lanes
                        // hold different cells, so they add into different nodes, and no lane reads a node another
                        // lane is still writing (a lane's next node may be its neighbour's current one)
                        float4* r3 = pwin + fu_node(lx, ly + oy, lz + oz);
#pragma unroll
                        for (int ox = 0; ox < 3; ox++) {
                            __syncwarp();
                            if (nagg > 0) {
                                float4 t = r3[ox];
                                t.x += a01[ox].x;
                                t.y += a01[ox].y;
                                t.z += a23[ox].x;
                                t.w += a23[ox].y;
                                r3[ox] = t;
                            }
                        }
                    }
                }
                __syncwarp();
                if (nagg > 0) {
                    atomicAdd(s.cell_count + key0 + c, nagg);
                    stayed += nagg;
                }
            }
            __syncthreads();   // the list is free for the next batch of rounds
            r0 = r;
        }
        // the unit's particles that stayed all count toward brick b
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) stayed += __shfl_xor_sync(0xffffffffu, stayed, o);
        if (lane == 0 && stayed) atomicAdd(brick_n, stayed);
        __syncthreads();
        if (tid == 0 && *brick_n) atomicAdd(s.brick_count + b, *brick_n);
        // 4. the warps' windows summed, and the touched nodes added into grid k+1
        for (int i = tid; i < WN; i += T) {
            float4 t = pwin_all[i];
#pragma unroll
            for (int w = 1; w < NW; w++) {
                const float4 q = pwin_all[w * WN + i];
                t.x += q.x;
                t.y += q.y;
                t.z += q.z;
                t.w += q.w;
            }
            if (t.x == 0.0f && t.y == 0.0f && t.z == 0.0f && t.w == 0.0f) continue;
            const int x = i % WIN, y = (i / WIN) % WIN, z = i / (WIN * WIN);
            const int gx = cx0 + x, gy = cy0 + y, gz = cz0 + z;
            if (gx >= dm.nx || gy >= dm.ny || gz >= dm.nz) {
                set_status(s.status, ST_OOB);
                continue;
            }
            red_add_v4(grid_out + ((int64_t)gz * dm.ny + gy) * dm.nx + gx, t.x, t.y, t.z, t.w);
        }
        __syncthreads();
    }
}

#ifndef VF_FUSED_CHUNK
#define VF_FUSED_CHUNK 2
#endif
#ifndef VF_FUSED_DEPTH
#define VF_FUSED_DEPTH 2
#endif
constexpr int FU_K = VF_FUSED_CHUNK;    // particles a chunk (a build may choose another)
constexpr int FU_UZ = VF_FUSED_DEPTH;   // unit depth in cells: 2 (128 threads) or 4 (256 threads)

cudaError_t fused_prepare() {
    return cudaFuncSetAttribute(k_g2p2g3<FU_UZ, FU_K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)FusedUnit<FU_UZ>::SMEM);
}

int fused_blocks_per_sm() { return FU_UZ == 4 ? 2 : 4; }

cudaError_t launch_g2p2g3(int blocks, const Step3& s, float4* grid_out, cudaStream_t stream) {
    k_g2p2g3<FU_UZ, FU_K><<<blocks, FusedUnit<FU_UZ>::T, FusedUnit<FU_UZ>::SMEM, stream>>>(s, grid_out);
    return cudaGetLastError();
}

}  // namespace vf
