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
    warp_tally(s.cell_count, key, valid, s.nkeys, s.status);
    warp_tally(s.brick_count, key >> 9, valid, s.nbricks, s.status);
    if (valid) s.key[i] = key;
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

// ------------------------------------------------------------------ P2G: exact fixed point

__device__ __forceinline__ long long fixed3(float v) {
    return __float2ll_rn(__fmul_rn(v, (float)(1ull << FIXED3_BITS)));
}

// One thread per particle; Flip3.scatter's amounts (Flip3.java:193-246) with every operation rounded on its own
// (__f*_rn: the compiler may not contract them), as the oracle computes them.
__global__ void __launch_bounds__(256) k_p2g3_fixed(Step3 s, unsigned long long* q) {
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
    const int64_t nodes = (int64_t)nx * ny * s.d.nz;
    const int64_t base = ((int64_t)cell[2] * ny + cell[1]) * nx + cell[0];
    const long long mass = fixed3(m);
    long long rest = mass;
#pragma unroll
    for (int k = 0; k < 27; k++) {
        const int ox = k % 3, oy = (k / 3) % 3, oz = k / 9;
        const float wgt = __fmul_rn(w[0][ox], __fmul_rn(w[1][oy], w[2][oz]));
        const float dd[3] = {__fsub_rn((float)ox, off[0]), __fsub_rn((float)oy, off[1]), __fsub_rn((float)oz, off[2])};
        const float wm = __fmul_rn(wgt, m);
        const int64_t node = base + (int64_t)oz * nx * ny + oy * nx + ox;
        if (k != 13) {   // the centre node (1, 1, 1) takes the rest below
            const long long share = fixed3(wm);
            rest -= share;
            atomicAdd(q + node, (unsigned long long)share);
        }
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const float at3 = __fadd_rn(vel[a], __fadd_rn(__fmul_rn(c[3 * a], dd[0]),
                                                          __fadd_rn(__fmul_rn(c[3 * a + 1], dd[1]),
                                                                    __fmul_rn(c[3 * a + 2], dd[2]))));
            const float push = __fmul_rn(sp, dd[a]);
            const float mom = __fadd_rn(__fmul_rn(wm, at3), __fmul_rn(wgt, push));
            atomicAdd(q + (int64_t)(1 + a) * nodes + node, (unsigned long long)fixed3(mom));
        }
    }
    atomicAdd(q + base + (int64_t)nx * ny + nx + 1, (unsigned long long)rest);
}

__global__ void k_fixed_to_grid3(const long long* q, float4* grid, int64_t nodes) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nodes) return;
    const double inv = 1.0 / (double)(1ull << FIXED3_BITS);
    grid[i] = make_float4(__double2float_rn(__ll2double_rn(q[i]) * inv), __double2float_rn(__ll2double_rn(q[nodes + i]) * inv),
                          __double2float_rn(__ll2double_rn(q[2 * nodes + i]) * inv),
                          __double2float_rn(__ll2double_rn(q[3 * nodes + i]) * inv));
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

// Each warp takes work units of (non-empty brick, 8 x 8 x UZ cells), 8 / UZ per brick, with no barrier between warps.
//
//  1. A unit's 64 UZ cells are consecutive keys, so their particle runs form one contiguous range of the sort's
//     permutation. The warp stages it in shared memory, puts each cell's run in ascending order there (the stable
//     sort's fix-up, fused here: G2P then reads the stable permutation), and writes the range back.
//  2. The unit's non-empty cells, ordered by particle count (largest first), go to the lanes in rounds of 32: a lane
//     sums one whole cell's 27 x 4 deposits in registers (loading two particles ahead), and when the round's fullest
//     cell is done all its lanes add their sums into the warp's 10 x 10 x (UZ + 2) node window in shared memory at
//     once. A cell's count varies (about 8 +- 2.6 at 8 per cell); the ordering puts cells of like counts in one
//     round, so few lanes wait. A round's lanes hold distinct cells, so at one stencil offset they add into distinct
//     nodes: plain read-modify-writes, a warp sync between offsets. (Dealing cells from a queue instead, each lane
//     taking the next cell as soon as its own was done, measured 1.3x slower at 8.2M particles: its lanes added
//     into the window at scattered times, and that divergent add ran nearly every iteration.)
//  3. The warp reduces every touched node of its window into the grid with one 16-byte vector
//     reduction (red.global.add.v4.f32); neighbouring units' windows overlap, and the reductions add.
//
// The per-particle arithmetic is Flip3.scatter's regrouped so a node costs a weight, one mass FMA and
// three momentum FMAs:  momentum_a(node o) = w(o) (A_a + sum_e B_ae o_e),
//   A_a = m (v_a - sum_e C_ae f_e) - s f_a,  B_ae = m C_ae + s [a == e],
// which is (w m)(v_a + C_a . d) + w s d_a with d = o - f (Flip3.java:225-243).
constexpr int P2G_THREADS = 128;
constexpr int P2G_WARPS = P2G_THREADS / 32;
// A work unit is UZ brick z-layers. One layer (8x8x1 cells, about 500 particles at 8 a cell) measured fastest at
// every size: 0.54x the time of two layers at 17k particles, 0.91x at 2.9M, 0.95x at 7.2M (more units even out
// the warps' loads and shorten their tails). Deeper units measured slower (4 layers: 2.6x at 8.2M).
constexpr int WWX = WIN, WWY = WIN;
constexpr int RUN_CAP = 2048;   // particle slots of one unit staged in shared memory (more: sorted in place)
constexpr int NBUCKET = 32;     // count buckets of the cell order (counts of 31 and more share the last)

template <int UZ>
struct P2GUnit {
    static constexpr int UCELLS = BRICK * BRICK * UZ;            // 64 UZ cells
    static constexpr int UPB = BRICK / UZ;                       // units per brick
    static constexpr int WWZ = UZ + 2, WW = WWX * WWY * WWZ;     // a warp's window: 100 (UZ + 2) nodes
};

template <int UZ>
struct P2GShared {
    float4 wwin[P2G_WARPS][P2GUnit<UZ>::WW];
    int run[P2G_WARPS][RUN_CAP];         // the unit's range of the permutation, sorted per cell here
    int start[P2G_WARPS][P2GUnit<UZ>::UCELLS + 1];    // cell c's particles: [start[c], start[c + 1])
    unsigned char order[P2G_WARPS][P2GUnit<UZ>::UCELLS];   // non-empty cells by descending count
    int bucket[P2G_WARPS][NBUCKET];
};
// One particle's fields, as the scatter reads them.
struct PIn {
    float x, y, z, u, v, w, m, j, c[9];
};

__device__ __forceinline__ void load_pin(PIn& q, const float* __restrict__ in, int64_t st, int src) {
    const float* b = in + src;
    q.x = b[X * st];
    q.y = b[Y * st];
    q.z = b[Z * st];
    q.u = b[U * st];
    q.v = b[V * st];
    q.w = b[W * st];
    q.m = b[M * st];
    q.j = b[J * st];
#pragma unroll
    for (int a = 0; a < 9; a++) q.c[a] = b[(C00 + a) * st];
}

__device__ __forceinline__ int checked_src(const int* run, int i, int np, uint32_t* status) {
    int src = run[i];
    if ((unsigned)src >= (unsigned)np) {
        set_status(status, ST_OOB);
        src = 0;
    }
    return src;
}

template <int UZ>
__global__ void __launch_bounds__(P2G_THREADS, 2) k_p2g3_tile(Step3 s) {
    constexpr int UCELLS = P2GUnit<UZ>::UCELLS, UPB = P2GUnit<UZ>::UPB, WW = P2GUnit<UZ>::WW;
    extern __shared__ __align__(16) unsigned char p2g_raw[];
    P2GShared<UZ>& S = *reinterpret_cast<P2GShared<UZ>*>(p2g_raw);
    const Params3 p = *s.params;
    const float vol = __fdiv_rn(1.0f, p.rho0);                 // V0 = m / rho0 as m * (1/rho0)
    const float k4dt = 4.0f * p.dt;
    const Dims3 dm = s.d;
    const int64_t st = s.stride;
    const float* __restrict__ in = s.in;
    int* __restrict__ perm = s.perm;
    const unsigned ALL = 0xffffffffu;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float4* ww = S.wwin[warp];
    int* cstart = S.start[warp];
    unsigned char* order = S.order[warp];
    int* bucket = S.bucket[warp];
    const int units = *s.n_active * UPB;
    const int total_warps = gridDim.x * P2G_WARPS;
    for (int u = blockIdx.x * P2G_WARPS + warp; u < units; u += total_warps) {
        const int b = s.active[u / UPB], lz0 = (u % UPB) * UZ;
        const int bx = b % dm.nbx, by = (b / dm.nbx) % dm.nby, bz = b / (dm.nbx * dm.nby);
        const int cx0 = bx * BRICK, cy0 = by * BRICK, cz0 = bz * BRICK + lz0;
        int bs = s.brick_start[b], be = s.brick_start[b + 1];
        if (bs < 0 || be > s.np || be < bs) {
            set_status(s.status, ST_OOB);
            bs = max(bs, 0);
            be = min(max(be, bs), s.np);
        }
        // the unit's cell starts (clamped into the brick and made non-decreasing)
        const int64_t key0 = (int64_t)b * 512 + lz0 * 64;
        for (int c = lane; c <= UCELLS; c += 32) {
            int v = (c < UCELLS || lz0 + UZ < BRICK) ? s.cell_start[key0 + c] : be;
            if (v < bs || v > be) {
                set_status(s.status, ST_OOB);
                v = min(max(v, bs), be);
            }
            cstart[c] = v;
        }
        __syncwarp();
        // a prefix maximum keeps the runs ordered even if the starts were not
        int carry = bs;
        for (int c0 = 0; c0 <= UCELLS; c0 += 32) {
            const int c = c0 + lane;
            int v = c <= UCELLS ? cstart[c] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(ALL, v, o);
                if (lane >= o) v = max(v, y);
            }
            v = max(v, carry);
            if (c <= UCELLS) cstart[c] = v;
            carry = __shfl_sync(ALL, v, 31);
        }
        __syncwarp();
        const int S0 = cstart[0], S1 = cstart[UCELLS];
        if (S1 == S0) continue;   // an empty unit (warp-uniform)

        // 1. the unit's range staged, each cell's run sorted there, written back
        const bool staged = S1 - S0 <= RUN_CAP;
        int* rs = S.run[warp];
        if (staged) {
            for (int j = S0 + lane; j < S1; j += 32) rs[j - S0] = perm[j];
            __syncwarp();
            for (int c = lane; c < UCELLS; c += 32)
                if (cstart[c + 1] - cstart[c] > 1) insertion_sort_run(rs + (cstart[c] - S0), cstart[c + 1] - cstart[c]);
            __syncwarp();
            for (int j = S0 + lane; j < S1; j += 32) perm[j] = rs[j - S0];
        } else {
            for (int c = lane; c < UCELLS; c += 32)
                if (cstart[c + 1] - cstart[c] > 1) insertion_sort_run(perm + cstart[c], cstart[c + 1] - cstart[c]);
        }
        const int* run = staged ? rs : perm + S0;   // the range, indexed from S0

        // the order: non-empty cells by count, largest first, ascending cell within a count
        bucket[lane] = 0;
        for (int j = lane; j < WW; j += 32) ww[j] = make_float4(0, 0, 0, 0);
        __syncwarp();
        for (int c = lane; c < UCELLS; c += 32) {
            const int n = cstart[c + 1] - cstart[c];
            if (n > 0) atomicAdd(&bucket[NBUCKET - 1 - min(n, NBUCKET - 1)], 1);
        }
        __syncwarp();
        int ncells;
        {
            int v = bucket[lane], x = v;   // exclusive scan over the buckets (largest counts first)
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(ALL, x, o);
                if (lane >= o) x += y;
            }
            bucket[lane] = x - v;
            ncells = __shfl_sync(ALL, x, 31);   // the number of non-empty cells
        }
        __syncwarp();
        for (int c0 = 0; c0 < UCELLS; c0 += 32) {   // UCELLS is a multiple of 32
            const int c = c0 + lane;
            const int n = cstart[c + 1] - cstart[c];
            const int key = n > 0 ? NBUCKET - 1 - min(n, NBUCKET - 1) : -1;
            const unsigned peers = __match_any_sync(ALL, key);
            const int base = key >= 0 ? bucket[key] : 0;
            __syncwarp();
            if (key >= 0) {
                order[base + __popc(peers & ((1u << lane) - 1))] = (unsigned char)c;
                if ((peers & ((1u << lane) - 1)) == 0) bucket[key] = base + __popc(peers);
            }
            __syncwarp();
        }

        // 2. the cells in rounds of 32 lanes, fullest first: a lane sums one cell's 27 x 4
        // deposits in registers; a round's cells have similar counts, so its lanes finish together and add into the
        // window together (distinct cells: distinct nodes at each stencil offset, a warp barrier between offsets)
        float2 acc01[27], acc23[27];   // per node (mass, x-momentum) and (y-, z-momentum)
        for (int r0 = 0; r0 < ncells; r0 += 32) {
#pragma unroll
            for (int k = 0; k < 27; k++) acc01[k] = acc23[k] = make_float2(0.0f, 0.0f);
            const int cell = r0 + lane < ncells ? order[r0 + lane] : -1;
            int i = 0, end = 0;
            PIn nxt, nxt2;
            if (cell >= 0) {
                i = cstart[cell];
                end = cstart[cell + 1];
                load_pin(nxt, in, st, checked_src(run, i - S0, s.np, s.status));
                if (i + 1 < end) load_pin(nxt2, in, st, checked_src(run, i + 1 - S0, s.np, s.status));
            }
            const int steps = (int)__reduce_max_sync(ALL, (unsigned)(end - i));
            for (int t = 0; t < steps; t++) {
                if (i < end) {
                    const PIn qq = nxt;
                    nxt = nxt2;
                    if (i + 2 < end) load_pin(nxt2, in, st, checked_src(run, i + 2 - S0, s.np, s.status));
                    i++;
                    int cl[3];
                    float f[3];
                    stencil_axis(qq.x, dm.nx, cl[0], f[0]);
                    stencil_axis(qq.y, dm.ny, cl[1], f[1]);
                    stencil_axis(qq.z, dm.nz, cl[2], f[2]);
                    const bool mine = cl[0] == cx0 + (cell & 7) && cl[1] == cy0 + ((cell >> 3) & 7) && cl[2] == cz0 + (cell >> 6);
                    if (!mine) set_status(s.status, ST_OOB);
                    if (mine && qq.m > 0.0f) {
                        float wx[3], wy[3], wz[3];
    #pragma unroll
                        for (int e = 0; e < 3; e++) {
                            float* we = e == 0 ? wx : e == 1 ? wy : wz;
                            const float ta = 1.5f - f[e], tc = f[e] - 1.0f, te = f[e] - 0.5f;
                            we[0] = 0.5f * (ta * ta);
                            we[1] = 0.75f - tc * tc;
                            we[2] = 0.5f * (te * te);
                        }
                        float jp;
                        if (p.tait) {
                            const float r = __frcp_rn(qq.j), r2 = r * r;
                            jp = p.bulk * ((r2 * r2) * r2 - qq.j);
                        } else {
                            jp = p.bulk * (1.0f - qq.j);
                        }
                        const float sp = (k4dt * (qq.m * vol)) * jp;
                        const float vel[3] = {qq.u, qq.v, qq.w};
                        float A[3], B[3][3];
    #pragma unroll
                        for (int r = 0; r < 3; r++) {
                            const float c0 = qq.c[3 * r], c1 = qq.c[3 * r + 1], c2 = qq.c[3 * r + 2];
                            A[r] = qq.m * (vel[r] - (c0 * f[0] + c1 * f[1] + c2 * f[2])) - sp * f[r];
                            B[r][0] = qq.m * c0;
                            B[r][1] = qq.m * c1;
                            B[r][2] = qq.m * c2;
                            B[r][r] += sp;
                        }
                        // paired fp32 (FFMA2): a node's (mass, x-momentum) += wx (m wyz, wyz M_x) and (y-, z-momentum)
                        // += wx (wyz M_y, wyz M_z), M_a = T_a + ox B_a0, T_a = A_a + oy B_a1 + oz B_a2; the mass lane
                        // rides along with zero coefficients
                        const float2 c01 = make_float2(qq.m, A[0]), c23 = make_float2(A[1], A[2]);
                        const float2 b0_01 = make_float2(0.0f, B[0][0]), b0_23 = make_float2(B[1][0], B[2][0]);
                        const float2 b1_01 = make_float2(0.0f, B[0][1]), b1_23 = make_float2(B[1][1], B[2][1]);
                        const float2 b2_01 = make_float2(0.0f, B[0][2]), b2_23 = make_float2(B[1][2], B[2][2]);
    #pragma unroll
                        for (int oz = 0; oz < 3; oz++) {
    #pragma unroll
                            for (int oy = 0; oy < 3; oy++) {
                                const float wyz = wy[oy] * wz[oz];
                                const float2 w2 = make_float2(wyz, wyz);
                                float2 t01 = c01, t23 = c23;
                                if (oy) {
                                    const float2 f2 = make_float2((float)oy, (float)oy);
                                    t01 = __ffma2_rn(f2, b1_01, t01);
                                    t23 = __ffma2_rn(f2, b1_23, t23);
                                }
                                if (oz) {
                                    const float2 f2 = make_float2((float)oz, (float)oz);
                                    t01 = __ffma2_rn(f2, b2_01, t01);
                                    t23 = __ffma2_rn(f2, b2_23, t23);
                                }
                                const float2 g01 = __fmul2_rn(w2, t01), g23 = __fmul2_rn(w2, t23);
                                const float2 h01 = __fmul2_rn(w2, b0_01), h23 = __fmul2_rn(w2, b0_23);
    #pragma unroll
                                for (int ox = 0; ox < 3; ox++) {
                                    const int kk = (oz * 3 + oy) * 3 + ox;
                                    float2 q01 = g01, q23 = g23;
                                    if (ox == 1) {
                                        q01 = __fadd2_rn(q01, h01);
                                        q23 = __fadd2_rn(q23, h23);
                                    } else if (ox == 2) {
                                        const float2 two = make_float2(2.0f, 2.0f);
                                        q01 = __ffma2_rn(two, h01, q01);
                                        q23 = __ffma2_rn(two, h23, q23);
                                    }
                                    const float2 x2 = make_float2(wx[ox], wx[ox]);
                                    acc01[kk] = __ffma2_rn(x2, q01, acc01[kk]);
                                    acc23[kk] = __ffma2_rn(x2, q23, acc23[kk]);
                                }
                            }
                        }
                    }

                }
            }
            const unsigned fm = __ballot_sync(ALL, cell >= 0);
            if (cell >= 0) {
                const int wb = ((cell >> 6) * WWY + ((cell >> 3) & 7)) * WWX + (cell & 7);
#pragma unroll
                for (int k = 0; k < 27; k++) {
                    const int ox = k % 3, oy = (k / 3) % 3, oz = k / 9;
                    const int wi = wb + (oz * WWY + oy) * WWX + ox;
                    float4 v = ww[wi];
                    v.x += acc01[k].x;
                    v.y += acc01[k].y;
                    v.z += acc23[k].x;
                    v.w += acc23[k].y;
                    ww[wi] = v;
                    __syncwarp(fm);
                }
            }
            __syncwarp();
        }
        __syncwarp();
        // 3. the window's touched nodes into the grid
        for (int j = lane; j < WW; j += 32) {
            const float4 t = ww[j];
            if (t.x == 0.0f && t.y == 0.0f && t.z == 0.0f && t.w == 0.0f) continue;
            const int gx = cx0 + j % WWX, gy = cy0 + (j / WWX) % WWY, gz = cz0 + j / (WWX * WWY);
            if (gx >= dm.nx || gy >= dm.ny || gz >= dm.nz) {
                set_status(s.status, ST_OOB);
                continue;
            }
            float4* node = node_addr(s, gx, gy, gz);
            if (!node) {
                set_status(s.status, ST_POOL);
                continue;
            }
            red_add_v4(node, t.x, t.y, t.z, t.w);
        }
        __syncwarp();
    }
}

constexpr int P2G_UZ = 1;   // the unit depth the scatter runs

size_t p2g_tile_smem() { return sizeof(P2GShared<P2G_UZ>); }

cudaError_t p2g_tile_prepare() {
    return cudaFuncSetAttribute(k_p2g3_tile<P2G_UZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)p2g_tile_smem());
}

cudaError_t launch_p2g3_tile(int blocks, const Step3& s, cudaStream_t stream) {
    k_p2g3_tile<P2G_UZ><<<blocks, P2G_THREADS, p2g_tile_smem(), stream>>>(s);
    return cudaGetLastError();
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
    warp_tally(s.cell_count, key, valid, s.nkeys, s.status);
    warp_tally(s.brick_count, key >> 9, valid, s.nbricks, s.status);
    if (valid) s.key[d] = key;
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

// Work items are bricks (or, in scenes of few bricks, slices of a brick's particles), taken by the CTAs from a
// counter in device memory (s.work, zeroed by the sort's brick scan): a CTA that finishes a small brick takes the
// next one, so the kernel ends when the work does rather than when the CTA dealt the most bricks does. A CTA
// takes its next item while it gathers the current one, and reads that item's brick and particle range then too.
//
// Per item the brick's 10^3 node window is read once from HBM and turned into velocities in shared memory (the grid
// update, Flip3.grid, fused: no velocity grid in HBM); the window's node loads are issued together, and the item's
// first particles' permutation entries and fields are requested before the window is computed, so the item starts
// after about two memory round trips. Then each particle of the brick gathers its 27 nodes from shared memory.
// The gather is regrouped per row of three nodes along x:
//   r0_a = sum_ox wx v_a,  rx_a = wx1 v_a(1) + 2 wx2 v_a(2),
//   vel_a = sum wyz r0_a,  S_ax = sum wyz rx_a,  S_ay = sum oy wyz r0_a,  S_az = sum oz wyz r0_a,
//   C_ae = 4 (S_ae - f_e vel_a)      (= 4 sum w v_a (o_e - f_e), Flip3.java:349-365).
constexpr int G2P_THREADS = 256;
constexpr int G2P_WLOADS = (WIN3 + G2P_THREADS - 1) / G2P_THREADS;   // window nodes a thread loads

// An item's brick and particle range, clamped into [0, np].
struct G2PItem {
    int b, bs, be;
};

__device__ __forceinline__ G2PItem g2p_item(const Step3& s, int a, int split) {
    G2PItem t;
    t.b = s.active[a / split];
    int bs = s.brick_start[t.b], be = s.brick_start[t.b + 1];
    if (bs < 0 || be > s.np || be < bs) {
        set_status(s.status, ST_OOB);
        bs = max(bs, 0);
        be = min(max(be, bs), s.np);
    }
    if (split > 1) {   // this item's slice of the brick's particles
        const int part = a % split;
        const int64_t len = be - bs;
        const int e = bs + (int)(len * (part + 1) / split);
        bs = bs + (int)(len * part / split);
        be = e;
    }
    t.bs = bs;
    t.be = be;
    return t;
}

__global__ void __launch_bounds__(G2P_THREADS, 4) k_g2p3_tile(Step3 s) {
    __shared__ float4 vwin[WIN3];
    __shared__ int4 next_item[2];   // {item, brick, start, end} of a CTA's next item, double-buffered
    const Params3 p = *s.params;
    const Dims3 dm = s.d;
    const int64_t st = s.stride;
    const int tid = threadIdx.x;
    const int split = max(s.g2p_split, 1);
    const int items = *s.n_active * split;
    if (tid == 0) {
        const int a = atomicAdd(s.work, 1);
        int4 v = make_int4(a, 0, 0, 0);
        if (a < items) {
            const G2PItem t = g2p_item(s, a, split);
            v = make_int4(a, t.b, t.bs, t.be);
        }
        next_item[0] = v;
    }
    __syncthreads();
    for (int slot = 0;; slot ^= 1) {
        const int4 cur = next_item[slot];
        if (cur.x >= items) break;   // uniform: every thread read the same entry after a barrier
        // the next item, claimed now and read while this one is gathered
        int nxt = 0;
        if (tid == 0) nxt = atomicAdd(s.work, 1);
        const int b = cur.y, bs = cur.z, be = cur.w;
        const int bx = b % dm.nbx, by = (b / dm.nbx) % dm.nby, bz = b / (dm.nbx * dm.nby);
        const int cx0 = bx * BRICK, cy0 = by * BRICK, cz0 = bz * BRICK;
        // the window's node loads, all issued before any is used
        float4 raw[G2P_WLOADS];
        bool have[G2P_WLOADS];
#pragma unroll
        for (int q = 0; q < G2P_WLOADS; q++) {
            const int wi = tid + q * G2P_THREADS;
            const int gx = cx0 + wi % WIN, gy = cy0 + (wi / WIN) % WIN, gz = cz0 + wi / (WIN * WIN);
            raw[q] = make_float4(0, 0, 0, 0);
            have[q] = false;
            if (wi < WIN3 && gx < dm.nx && gy < dm.ny && gz < dm.nz) {
                if (s.vel_ready) {
                    raw[q] = s.vel[((int64_t)gz * dm.ny + gy) * dm.nx + gx];
                    have[q] = true;
                } else if (const float4* node = node_addr(s, gx, gy, gz)) {
                    raw[q] = *node;
                    have[q] = true;
                } else {
                    set_status(s.status, ST_POOL);
                }
            }
        }
        // Every thread walks the same number of iterations so the warp-level count is converged. The
        // permutation is read two iterations ahead and the particle one iteration ahead of its use.
        const int iters = (be - bs + G2P_THREADS - 1) / G2P_THREADS;
        const int d0 = bs + tid;
        auto src_of = [&](int d) {
            int v = d < be ? (s.perm ? s.perm[d] : d) : -1;
            if (d < be && (unsigned)v >= (unsigned)s.np) {
                set_status(s.status, ST_OOB);
                v = -1;
            }
            return v;
        };
        int src_a = src_of(d0);
        int src_b = src_of(d0 + G2P_THREADS);
        float nx_ = 0, ny_ = 0, nz_ = 0, nm_ = 0, nj_ = 0;
        if (src_a >= 0) {
            nx_ = s.in[X * st + src_a];
            ny_ = s.in[Y * st + src_a];
            nz_ = s.in[Z * st + src_a];
            nm_ = s.in[M * st + src_a];
            nj_ = s.in[J * st + src_a];
        }
        // the window's velocities
#pragma unroll
        for (int q = 0; q < G2P_WLOADS; q++) {
            const int wi = tid + q * G2P_THREADS;
            if (wi < WIN3) {
                float4 v = make_float4(0, 0, 0, 0);
                if (have[q]) {
                    if (s.vel_ready) {
                        v = raw[q];
                    } else {
                        const int gx = cx0 + wi % WIN, gy = cy0 + (wi / WIN) % WIN, gz = cz0 + wi / (WIN * WIN);
                        const float3 u = grid_velocity(raw[q], gx, gy, gz, dm, p);
                        v = make_float4(u.x, u.y, u.z, 0.0f);
                    }
                }
                vwin[wi] = v;
            }
        }
        if (tid == 0) {   // the next item's brick and range (its claim has had the window loads' time to return)
            int4 v = make_int4(nxt, 0, 0, 0);
            if (nxt < items) {
                const G2PItem t = g2p_item(s, nxt, split);
                v = make_int4(nxt, t.b, t.bs, t.be);
            }
            next_item[slot ^ 1] = v;
        }
        __syncthreads();
        for (int it = 0; it < iters; it++) {
            const int d = d0 + it * G2P_THREADS;
            const bool valid = d < be && src_a >= 0;
            const int src = src_a;
            const float at[3] = {nx_, ny_, nz_};
            const float m = nm_, jold = nj_;
            if (src_b >= 0) {
                nx_ = s.in[X * st + src_b];
                ny_ = s.in[Y * st + src_b];
                nz_ = s.in[Z * st + src_b];
                nm_ = s.in[M * st + src_b];
                nj_ = s.in[J * st + src_b];
            }
            src_a = src_b;
            src_b = src_of(d + 2 * G2P_THREADS);
            float pos[3] = {0, 0, 0};
            if (valid) {
                if (!(m > 0.0f)) {
                    g2p_copy(s, d, src, pos);
                } else {
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
                        float j = jold * (1.0f + p.dt * (c[0] + (c[4] + c[8])));
                        j = clampf(j, 1.0f / J_BOUND3, J_BOUND3);
                        g2p_store(s, d, pos, vel, c, m, j);
                    }
                }
            }
            g2p_count(s, d, valid, pos);
        }
        __syncthreads();   // the window is free, and next_item[slot ^ 1] is visible
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

__global__ void __launch_bounds__(256) k_min_positive3(const float* m, int n, unsigned* out) {
    unsigned best = 0x7f7fffffu;   // FLT_MAX
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float v = m[i];
        if (v > 0.0f) best = min(best, __float_as_uint(v));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0 && best != 0x7f7fffffu) atomicMin(out, best);
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
