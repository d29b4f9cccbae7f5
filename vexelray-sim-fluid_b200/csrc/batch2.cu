// batch2.cu -- many independent 2D scenes (each a FlipStep: sort by cell, scatter, grid, advect;
// FlipStep.java:81-193, Flip.java) stepped by ONE cooperative persistent kernel launch per step,
// the launches replayed from a CUDA graph. No counterpart in the reference, which steps one scene
// per ParticleSimulation; the per-particle and per-node arithmetic is the single-scene step's
// (mpm2_device.cuh), so each scene computes what vf_mpm2 computes for it.
//
// Layout in HBM (scenes side by side, no per-scene allocation):
//   particles   two sets (ping-pong by step parity) of 10 SoA f32 fields x y u v m j c00 c01 c10 c11;
//               scene s owns slots [p0, p0 + np) of every field, and keeps them: the sort is by
//               (scene, tile, cell), so a scene's particles never leave its range
//   grid        two buffers (by step parity) of float4 {m, mu, mv, 0} per node; scene s's nodes at
//               g0 + j*nx + i
//   tiles       a scene's (nx-2) x (ny-2) stencil cells are cut into tiles of tx x ty cells, ntx x nty
//               of them; the tile entries of all scenes, each scene's followed by a sentinel, hold the
//               per-step counts and the run starts (by parity)
//   cells       cell keys tile-major: key = c0 + tile * tx*ty + (ly * tx + lx), one count and one cursor
//               per key
//
// One step = five phases separated by a grid-wide barrier (the launch is cooperative, so every CTA is
// resident; the barrier's wait is bounded and sets a status bit rather than hang):
//   1  tile scan     per scene: tile counts -> run starts (parity buffer), counts zeroed; each tile's run cut
//                    into chunks of at most CHUNK particles, counted per scene
//   2  cell scan     a warp per non-empty tile: cell counts -> cursors (cell starts), counts zeroed; CTA 0 lays
//                    the scenes' chunks out one after another
//   3  permute       per slot: perm[cursor[key]++] = slot, one cursor bump per run of equal keys of a warp. Within a
//                    cell the order is the atomics' (unspecified, as in the reference's CountingSort,
//                    SortTest.java:121-134); what the scatter needs is each cell's particles contiguous. The
//                    chunks enter the item list, and the other parity's grid is cleared over the windows of
//                    the tiles the previous step scattered into.
//   4  scatter       a warp per chunk, work-stealing: the tile's cells clipped to the chunk (the cursors hold
//                    each run's end) are ordered by count, largest first, and taken in rounds of 32, a lane a cell;
//                    a lane sums Flip.scatter's 27 amounts over its cell's particles in registers, and when the
//                    round's fullest cell is done all its lanes add their sums into the warp's private node window
//                    (a round's lanes hold distinct cells, so distinct nodes at each stencil offset: plain
//                    read-modify-write); then one 16-byte red.global.add.v4.f32 per touched window node
//   5  gather        a warp per chunk, work-stealing: the tile window's node velocities (Flip.grid, fused) into
//                    the warp's shared memory, then per particle Flip.advectBody; the particle is written to its
//                    sorted slot of the other set, and its next cell key tallied for the next step's sort.
// Chunks bound a work item, so a dense tile (tens of thousands of particles in the 64^2 scenes) spreads over
// many warps instead of one.
#include <algorithm>
#include <cmath>
#include <map>
#include <string>
#include <vector>

#include "mpm2_device.cuh"
#include "sort.cuh"

using namespace vf;

namespace {

struct Scene2 {
    int nx, ny, np;
    int tx, ty, ntx, nty, tc;   // tile shape in cells, tiles per axis, cells per tile
    int p0;                     // first particle slot
    int t0;                     // first tile entry: ntx*nty tiles, then a sentinel
    int c0;                     // first cell key
    int64_t g0;                 // first grid node
    Params2 prm;
};

// The batch's device state, passed by value to the step kernel.
struct Batch2 {
    const Scene2* scene;
    int nscenes;
    const int* tile_scene;     // tile entry -> scene, -1 for a sentinel
    int nentries;              // tile entries (every scene's tiles and its sentinel)
    float* part[2];
    int64_t stride;            // floats per field
    int np;                    // all scenes' particles
    int ncells;                // all scenes' cell keys
    int* key;                  // per slot of the current set: the cell key for this step's sort
    int* perm;                 // sorted slot -> slot of the current set
    int* cell_count;
    int* cursor;               // per cell: its run's start after the cell scan, its end after the permute
    int* tile_count;
    int* tile_start[2];        // per tile entry, by step parity: run start; the sentinel holds the scene's end
    int* chunk_start;          // per tile entry: its first chunk within its scene; the sentinel the scene's chunks
    int* scene_chunks;         // per scene: its chunks
    int* scene_chunk_start;    // per scene (and one past): its first chunk in the item list
    int4* item;                // per chunk: {tile entry, scene, first slot, end slot}, written by the permute phase
    int item_cap;              // item's length
    float4* grid[2];
    unsigned* step;            // device step counter (its parity picks the buffers)
    unsigned* work;            // work-stealing counters: [0] scatter, [1] gather
    GridBarrier* bar;
    int wmax;                  // window nodes of the largest tile (the shared-memory windows' stride)
    unsigned* done;            // CTAs finished with the launch (the last one closes the phase clock)
    unsigned long long* phase_ns;   // device time per phase summed over launches, the launch count, a stamp
    uint32_t* status;
};

constexpr int BATCH_MAX_THREADS = 512;
#ifndef BATCH_MIN_BLOCKS
#define BATCH_MIN_BLOCKS 1
#endif
constexpr int NPHASE = 5;         // tile scan, cell scan, permute, scatter, gather
constexpr int CHUNK = 1024;       // particles of a work item of the scatter and gather: a tile's run in chunks
// Shared memory of one warp of the step: its node window (m, mu, mv arrays of the largest tile's window; the
// gather reuses it for float2 velocities), then the scatter's cell queue: per cell of a tile (at most QCELLS) its
// particles' range within the chunk, the non-empty cells by descending count, count buckets, the queue's head.
constexpr int QCELLS = 512;                // cells of the largest tile (32 x 16)
constexpr int QBUCKETS = 32;               // count buckets (31 particles and more share the last)
constexpr int QWORDS = 2 * QCELLS + QCELLS / 2 + QBUCKETS + 4;   // a multiple of 4 words
__host__ __device__ constexpr int window_words(int wmax) { return (3 * wmax + 3) & ~3; }   // 16-byte aligned
__host__ __device__ constexpr int warp_smem_floats(int wmax) { return window_words(wmax) + QWORDS; }

// One particle's fields as the scatter reads them (source slot < 0: none, zeros).
struct Part2 {
    float x, y, u, v, m, j, c00, c01, c10, c11;
};

__device__ __forceinline__ void load_part2(Part2& q, const float* __restrict__ in, int64_t st, int src) {
    if (src < 0) {
        q = Part2{0, 0, 0, 0, 0, 1, 0, 0, 0, 0};
        return;
    }
    q.x = in[PX * st + src];
    q.y = in[PY * st + src];
    q.u = in[PU * st + src];
    q.v = in[PV * st + src];
    q.m = in[PM * st + src];
    q.j = in[PJ * st + src];
    q.c00 = in[PC00 * st + src];
    q.c01 = in[PC01 * st + src];
    q.c10 = in[PC10 * st + src];
    q.c11 = in[PC11 * st + src];
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// The next-step cell key and tile entry of a particle at (x, y) in scene sc.
__device__ __forceinline__ void batch_key(const Scene2& sc, float x, float y, int& key, int& tile) {
    int col, row;
    stencil_cell2(x, y, sc.nx, sc.ny, col, row);
    const int tix = col / sc.tx, tiy = row / sc.ty;
    const int local = tiy * sc.ntx + tix;
    tile = sc.t0 + local;
    key = sc.c0 + local * sc.tc + (row - tiy * sc.ty) * sc.tx + (col - tix * sc.tx);
}

__global__ void __launch_bounds__(BATCH_MAX_THREADS, BATCH_MIN_BLOCKS) k_batch2_step(Batch2 B) {
    extern __shared__ __align__(16) float dyn[];
    __shared__ int scan_smem[33];
    // a step after one whose grid barrier gave up does nothing: the barrier's count is no longer consistent
    __shared__ int dead;
    if (threadIdx.x == 0) dead = (*(volatile uint32_t*)B.status & ST_TIMEOUT) != 0;
    __syncthreads();
    if (dead) return;
    const unsigned par = *B.step & 1u;   // read before the first barrier; CTA 0 advances it after
    const float* __restrict__ in = B.part[par];
    float* __restrict__ out = B.part[par ^ 1u];
    int* ts_cur = B.tile_start[par];
    const int* ts_prev = B.tile_start[par ^ 1u];
    float4* g_cur = B.grid[par];
    float4* g_next = B.grid[par ^ 1u];
    const int64_t st = B.stride;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int gwarp = blockIdx.x * nwarps + warp, nwarps_all = gridDim.x * nwarps;
    float* ww = dyn + warp * warp_smem_floats(B.wmax);          // this warp's node window
    // the phase clock: CTA 0 stamps the start and every barrier, the last CTA to finish the end
    __shared__ unsigned long long stamp;
    if (blockIdx.x == 0 && threadIdx.x == 0) stamp = global_ns();
    auto phase_done = [&](int k) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            const unsigned long long now = global_ns();
            atomicAdd(&B.phase_ns[k], now - stamp);
            stamp = now;
            if (k == NPHASE - 2) B.phase_ns[NPHASE + 1] = now;   // the last phase's start
        }
    };

    // ---- 1. tile scan, per scene: tile counts -> run starts, and the tiles' chunks of <= CHUNK particles
    if (blockIdx.x == 0 && threadIdx.x == 0) B.work[1] = 0;   // the previous launch's gather counter
    for (int s = blockIdx.x; s < B.nscenes; s += gridDim.x) {
        const Scene2 sc = B.scene[s];
        const int nt = sc.ntx * sc.nty;
        int carry = 0, ccarry = 0;
        for (int base = 0; base < nt; base += blockDim.x) {
            const int i = base + threadIdx.x;
            const int c = i < nt ? B.tile_count[sc.t0 + i] : 0;
            int total, ctotal;
            const int ex = block_exclusive(c, scan_smem, &total);
            const int cex = block_exclusive((c + CHUNK - 1) / CHUNK, scan_smem, &ctotal);
            if (i < nt) {
                ts_cur[sc.t0 + i] = sc.p0 + carry + ex;
                B.chunk_start[sc.t0 + i] = ccarry + cex;
                B.tile_count[sc.t0 + i] = 0;
            }
            carry += total;
            ccarry += ctotal;
        }
        if (threadIdx.x == 0) {
            ts_cur[sc.t0 + nt] = sc.p0 + carry;
            B.chunk_start[sc.t0 + nt] = ccarry;
            B.scene_chunks[s] = ccarry;
            if (carry != sc.np) set_status(B.status, ST_RANK);
        }
    }
    if (!grid_barrier(B.bar, B.status)) return;
    phase_done(0);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(B.step, 1u);

    // ---- 2. cell scan, a warp per non-empty tile: the tile's cell counts -> cursors (cell starts); CTA 0 first
    // lays out the scenes' chunks one scene after another
    if (blockIdx.x == 0) {
        int carry = 0;
        for (int base = 0; base < B.nscenes; base += blockDim.x) {
            const int i = base + threadIdx.x;
            int total;
            const int ex = block_exclusive(i < B.nscenes ? B.scene_chunks[i] : 0, scan_smem, &total);
            if (i < B.nscenes) B.scene_chunk_start[i] = carry + ex;
            carry += total;
        }
        if (threadIdx.x == 0) B.scene_chunk_start[B.nscenes] = carry;
    }
    // The tiles, 32 at a time a warp: a lane reads one tile's run and scene (the reads of the warp's 32 tiles in
    // flight together); then the warp scans the non-empty ones one at a time, every lane on the tile's cells.
    for (int t0 = gwarp * 32; t0 < B.nentries; t0 += nwarps_all * 32) {
        const int tl = t0 + lane;
        const int sl = tl < B.nentries ? B.tile_scene[tl] : -1;
        int tsl = 0, tel = 0, tcl = 0, cbl = 0;
        bool live = false;
        if (sl >= 0) {
            tsl = ts_cur[tl];
            tel = ts_cur[tl + 1];
            const Scene2& sc = B.scene[sl];
            if (tel > tsl) {
                if (tsl < sc.p0 || tel > sc.p0 + sc.np) {   // counts that do not add up
                    set_status(B.status, ST_RANK);
                } else {
                    live = true;
                    tcl = sc.tc;                           // 64 .. 512 cells: 2 .. 16 per lane
                    cbl = sc.c0 + (tl - sc.t0) * sc.tc;
                }
            }
        }
        unsigned todo = __ballot_sync(0xffffffffu, live);
        while (todo) {
            const int l = __ffs(todo) - 1;
            todo &= todo - 1;
            const int ts = __shfl_sync(0xffffffffu, tsl, l), te = __shfl_sync(0xffffffffu, tel, l);
            const int tc = __shfl_sync(0xffffffffu, tcl, l);
            const int per = tc >> 5;
            const int cb = __shfl_sync(0xffffffffu, cbl, l) + lane * per;
            int c[16], sum = 0;
#pragma unroll
            for (int k = 0; k < 16; k++) {
                c[k] = k < per ? B.cell_count[cb + k] : 0;
                sum += c[k];
            }
            int run = ts + warp_inclusive(sum) - sum;
#pragma unroll
            for (int k = 0; k < 16; k++) {
                if (k < per) {
                    B.cursor[cb + k] = run;
                    B.cell_count[cb + k] = 0;
                    run += c[k];
                }
            }
            if (lane == 31 && run != te) set_status(B.status, ST_RANK);
        }
    }
    if (!grid_barrier(B.bar, B.status)) return;
    phase_done(1);

    // ---- 3. permute: perm[cursor[key]++] = slot, eight slots per thread, one cursor bump per run of equal keys of
    // a warp (the order within a cell is the atomics' order: unspecified, as in the reference's CountingSort); the
    // tiles' chunks entered in the item list; and the other parity's grid cleared over the windows of the tiles
    // the previous step scattered into
    {
        // PK slots a thread (a warp's slots consecutive), the next iteration's keys read while this one's atomics
        // are in flight
        constexpr int PK = 8;
        const int n32 = (B.np + 31) & ~31;
        const int stride = gridDim.x * blockDim.x;
        auto key_at = [&](int i) {
            int v = i < B.np ? B.key[i] : -1;
            if (i < B.np && (v < 0 || v >= B.ncells)) {
                set_status(B.status, ST_OOB);
                v = -1;
            }
            return v;
        };
        int kn[PK];
        const int first = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
        for (int u = 0; u < PK; u++) kn[u] = key_at(first + u * stride);
        for (int i0 = first; i0 < n32; i0 += PK * stride) {
            int k[PK];
#pragma unroll
            for (int u = 0; u < PK; u++) {
                k[u] = kn[u];
                kn[u] = key_at(i0 + (PK + u) * stride);
            }
            // the slots of a warp are consecutive, and in the last step's sorted order their keys come in runs:
            // one cursor bump per run of equal keys (a key in two runs of the warp takes two, with distinct ranks)
            int base[PK], rank[PK], leader[PK];
#pragma unroll
            for (int u = 0; u < PK; u++) {   // the atomics of the slots in flight together
                const int prev = __shfl_up_sync(0xffffffffu, k[u], 1);
                const unsigned starts = __ballot_sync(0xffffffffu, lane == 0 || prev != k[u]);
                leader[u] = 31 - __clz(starts & (0xffffffffu >> (31 - lane)));
                const unsigned above = starts & ~(0xffffffffu >> (31 - lane));
                const int end = above ? __ffs(above) - 1 : 32;
                rank[u] = lane - leader[u];
                base[u] = (lane == leader[u] && k[u] >= 0) ? atomicAdd(&B.cursor[k[u]], end - leader[u]) : 0;
            }
#pragma unroll
            for (int u = 0; u < PK; u++) {
                const int d = __shfl_sync(0xffffffffu, base[u], leader[u]) + rank[u];
                if (k[u] >= 0) {
                    if (d >= 0 && d < B.np) B.perm[d] = i0 + u * stride;
                    else set_status(B.status, ST_RANK);
                }
            }
        }
    }
    // The tiles, 32 at a time a warp, a lane a tile: each lane reads its tile's runs and scene (the reads of a warp's
    // 32 tiles in flight together) and enters the tile's chunks in the item list; then the warp clears, one tile at a
    // time with every lane on it, the windows of the tiles the previous step scattered into, from the lanes' values.
    for (int t0 = gwarp * 32; t0 < B.nentries; t0 += nwarps_all * 32) {
        const int t = t0 + lane;
        const int s = t < B.nentries ? B.tile_scene[t] : -1;
        int ts = 0, te = 0;
        bool clear = false;
        if (t < B.nentries) {
            ts = ts_cur[t];
            te = ts_cur[t + 1];
            clear = ts_prev[t + 1] > ts_prev[t];
        }
        int x0 = 0, y0 = 0, wx = 0, wn = 0, nxs = 0, nys = 0;
        int64_t g0 = 0;
        if (s >= 0) {
            const Scene2& sc = B.scene[s];
            if (te > ts && ts >= sc.p0 && te <= sc.p0 + sc.np) {   // the tile's chunks into the item list
                const int item0 = B.scene_chunk_start[s] + B.chunk_start[t];
                const int nch = (te - ts + CHUNK - 1) / CHUNK;
                for (int q = 0; q < nch; q++) {
                    if (item0 + q >= 0 && item0 + q < B.item_cap)
                        B.item[item0 + q] = make_int4(t, s, ts + q * CHUNK, min(te, ts + (q + 1) * CHUNK));
                    else set_status(B.status, ST_OOB);
                }
            }
            const int lt = t - sc.t0;
            x0 = (lt % sc.ntx) * sc.tx;
            y0 = (lt / sc.ntx) * sc.ty;
            wx = sc.tx + 2;
            wn = wx * (sc.ty + 2);
            nxs = sc.nx;
            nys = sc.ny;
            g0 = sc.g0;
        } else {
            clear = false;
        }
        unsigned todo = __ballot_sync(0xffffffffu, clear);
        while (todo) {
            const int l = __ffs(todo) - 1;
            todo &= todo - 1;
            const int cx0 = __shfl_sync(0xffffffffu, x0, l), cy0 = __shfl_sync(0xffffffffu, y0, l);
            const int cwx = __shfl_sync(0xffffffffu, wx, l), cwn = __shfl_sync(0xffffffffu, wn, l);
            const int cnx = __shfl_sync(0xffffffffu, nxs, l), cny = __shfl_sync(0xffffffffu, nys, l);
            const int64_t cg0 = __shfl_sync(0xffffffffu, g0, l);
            for (int j = lane; j < cwn; j += 32) {
                const int gi = cx0 + j % cwx, gj = cy0 + j / cwx;
                if (gi < cnx && gj < cny) g_next[cg0 + (int64_t)gj * cnx + gi] = make_float4(0, 0, 0, 0);
            }
        }
    }
    if (!grid_barrier(B.bar, B.status)) return;
    phase_done(2);
    const int items = min(B.scene_chunk_start[B.nscenes], B.item_cap);

    // ---- 4. scatter: each warp takes chunks (<= CHUNK particles of one tile) from the work counter and scatters
    // one alone through its own node window
    for (;;) {
        int k = 0;
        if (lane == 0) k = (int)atomicAdd(&B.work[0], 1u);
        k = __shfl_sync(0xffffffffu, k, 0);
        if (k >= items) break;
        const int4 it = B.item[k];   // the chunk: its tile entry, scene and slots
        const int t = it.x, s = it.y, c0 = it.z, c1 = it.w;
        if (t < 0 || t >= B.nentries || s < 0 || s >= B.nscenes) {
            if (lane == 0) set_status(B.status, ST_OOB);
            continue;
        }
        const Scene2& sc = B.scene[s];
        const int p0 = sc.p0, p1 = sc.p0 + sc.np;
        if (c0 >= c1 || c0 < p0 || c1 > p1) {
            if (lane == 0) set_status(B.status, ST_OOB);
            continue;
        }
        const int lt = t - sc.t0;
        const int tx = sc.tx, ty = sc.ty, nx = sc.nx, ny = sc.ny, tc = sc.tc;
        const int x0 = (lt % sc.ntx) * tx, y0 = (lt / sc.ntx) * ty;   // the tile's first cell = first node
        const int wx = tx + 2, wn = wx * (ty + 2);
        const Params2 prm = sc.prm;
        int2* crange = reinterpret_cast<int2*>(ww + window_words(B.wmax));   // per cell: its particles in the chunk
        unsigned short* order = reinterpret_cast<unsigned short*>(crange + QCELLS);
        int* bucket = reinterpret_cast<int*>(order + QCELLS);
        int* head = bucket + QBUCKETS;
        for (int j = lane; j < 3 * wn; j += 32) ww[j] = 0.0f;
        bucket[lane] = 0;
        __syncwarp();
        // the tile's cells (keys cb + j, j = ly * tx + lx; after the permute cursor[key] is the run's end) clipped
        // to the chunk, and counted into the buckets
        const int cb = sc.c0 + lt * tc;
        if (tc > QCELLS) {
            if (lane == 0) set_status(B.status, ST_OOB);
            continue;
        }
        for (int j = lane; j < tc; j += 32) {
            const int e = B.cursor[cb + j], b0 = j == 0 ? c0 : B.cursor[cb + j - 1];   // cell 0 starts at the tile's run start, <= c0
            const int lo = max(b0, c0), hi = min(e, c1);
            crange[j] = make_int2(lo, hi);
            if (hi > lo) atomicAdd(&bucket[QBUCKETS - 1 - min(hi - lo, QBUCKETS - 1)], 1);
        }
        __syncwarp();
        {
            const int v = bucket[lane];
            int x = v;   // exclusive scan over the buckets, largest counts first
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            bucket[lane] = x - v;
            if (lane == 31) *head = x;
        }
        __syncwarp();
        const int ncq = *head;   // non-empty cells
        for (int j = lane; j < tc; j += 32) {
            const int2 r = crange[j];
            if (r.y > r.x) order[atomicAdd(&bucket[QBUCKETS - 1 - min(r.y - r.x, QBUCKETS - 1)], 1)] = (unsigned short)j;
        }
        __syncwarp();
        // the non-empty cells in synchronous rounds of 32, fullest first: a lane sums its cell's 27 amounts
        // (Flip.scatter, Flip.java:269-303) over the cell's particles in registers; when the round's fullest cell is
        // done, all its lanes add their sums into the window at once. A round's cells have like counts, so few lanes
        // wait, and its lanes hold distinct cells, so at one stencil offset they write distinct nodes. (Dealing
        // cells from a queue, a lane taking the next cell when its own was done, left the window adds at scattered
        // times, divergent in nearly every iteration.)
        auto source = [&](int slot) {
            const int src = B.perm[slot];
            if (src < p0 || src >= p1) {
                set_status(B.status, ST_OOB);
                return -1;
            }
            return src;
        };
        float acc[27];
        for (int r0 = 0; r0 < ncq; r0 += 32) {
#pragma unroll
            for (int a = 0; a < 27; a++) acc[a] = 0.0f;
            const int cell = r0 + lane < ncq ? order[r0 + lane] : -1;
            int i = 0, end = 0;
            Part2 nxt, nxt2;   // the lane's next two particles in flight
            if (cell >= 0) {
                const int2 r = crange[cell];
                i = r.x;
                end = r.y;
                load_part2(nxt, in, st, source(i));
                if (i + 1 < end) load_part2(nxt2, in, st, source(i + 1));
            }
            const int steps = (int)__reduce_max_sync(0xffffffffu, (unsigned)max(end - i, 0));
            for (int n = 0; n < steps; n++) {
                if (i < end) {
                    const Part2 cur = nxt;
                    nxt = nxt2;
                    if (i + 2 < end) load_part2(nxt2, in, st, source(i + 2));
                    i++;
                    if (cur.m > 0.0f) {
                        const Stencil2 sn = stencil2(cur.x, cur.y, nx, ny);
                        if (sn.col == x0 + cell % tx && sn.row == y0 + cell / tx) {
                            const float sp = impulse_factor(prm.dt, cur.m, prm.rho0, prm.bulk, cur.j, prm.tait);
                            scatter_accumulate2(sn, cur.m, cur.u, cur.v, cur.c00, cur.c01, cur.c10, cur.c11, sp, acc);
                        } else {
                            set_status(B.status, ST_OOB);
                        }
                    }
                }
            }
            const unsigned fm = __ballot_sync(0xffffffffu, cell >= 0);
            if (cell >= 0) {
                const int wb = (cell / tx) * wx + cell % tx;
#pragma unroll
                for (int o = 0; o < 9; o++) {
                    const int wi = wb + (o / 3) * wx + o % 3;
                    ww[wi] += acc[3 * o];
                    ww[wn + wi] += acc[3 * o + 1];
                    ww[2 * wn + wi] += acc[3 * o + 2];
                    __syncwarp(fm);
                }
            }
            __syncwarp();   // this round's window writes before the next round's
        }
        __syncwarp();
        for (int j = lane; j < wn; j += 32) {
            const float a = ww[j], bu = ww[wn + j], bv = ww[2 * wn + j];
            if (a == 0.0f && bu == 0.0f && bv == 0.0f) continue;
            const int gi = x0 + j % wx, gj = y0 + j / wx;
            if (gi >= nx || gj >= ny) {
                set_status(B.status, ST_OOB);
                continue;
            }
            red_add_v4(&g_cur[sc.g0 + (int64_t)gj * nx + gi], a, bu, bv, 0.0f);
        }
        __syncwarp();   // the window is free for the next chunk
    }
    if (!grid_barrier(B.bar, B.status)) return;
    phase_done(3);
    if (blockIdx.x == 0 && threadIdx.x == 0) B.work[0] = 0;

    // ---- 5. gather: each warp takes chunks and gathers one alone: the tile window's node velocities (the grid
    // update) into its shared memory, then the chunk's particles advected
    float2* vw = reinterpret_cast<float2*>(ww);
    for (;;) {
        int k = 0;
        if (lane == 0) k = (int)atomicAdd(&B.work[1], 1u);
        k = __shfl_sync(0xffffffffu, k, 0);
        if (k >= items) break;
        const int4 it = B.item[k];   // the chunk: its tile entry, scene and slots
        const int t = it.x, s = it.y, c0 = it.z, c1 = it.w;
        if (t < 0 || t >= B.nentries || s < 0 || s >= B.nscenes) continue;   // flagged in the scatter
        const Scene2& sc = B.scene[s];
        const int p0 = sc.p0, p1 = sc.p0 + sc.np;
        if (c0 >= c1 || c0 < p0 || c1 > p1) continue;
        const int lt = t - sc.t0;
        const int tx = sc.tx, ty = sc.ty, nx = sc.nx, ny = sc.ny;
        const int x0 = (lt % sc.ntx) * tx, y0 = (lt / sc.ntx) * ty;
        const int wx = tx + 2, wn = wx * (ty + 2);
        const Params2 prm = sc.prm;
        for (int j = lane; j < wn; j += 32) {
            const int gi = x0 + j % wx, gj = y0 + j / wx;
            float2 v = make_float2(0.0f, 0.0f);
            if (gi < nx && gj < ny) {
                const float4 gv = g_cur[sc.g0 + (int64_t)gj * nx + gi];
                v = grid_velocity2(gv.x, gv.y, gv.z, gi, gj, nx, ny, prm);
            }
            vw[j] = v;
        }
        __syncwarp();
        // Groups of GG x 32 particles (GG a lane, 32 apart): a group's permutation entries are read two groups
        // ahead and its positions, J and masses one group ahead, so a lane has GG particles' loads in flight while
        // it advects the current group (a particle's arithmetic is far shorter than a load's round trip).
        constexpr int GG = 4;
        auto src_at = [&](int slot) {   // a sorted slot's source, checked (its own slot when out of range)
            if (slot >= c1) return -1;
            int v = B.perm[slot];
            if (v < p0 || v >= p1) {
                set_status(B.status, ST_OOB);
                v = slot;
            }
            return v;
        };
        int sa[GG], sb[GG];
        float qx[GG], qy[GG], qj[GG], qm[GG];
#pragma unroll
        for (int u = 0; u < GG; u++) {
            sa[u] = src_at(c0 + 32 * u + lane);
            sb[u] = src_at(c0 + 32 * (GG + u) + lane);
        }
#pragma unroll
        for (int u = 0; u < GG; u++) {
            qx[u] = qy[u] = qj[u] = qm[u] = 0.0f;
            if (sa[u] >= 0) {
                qx[u] = in[PX * st + sa[u]];
                qy[u] = in[PY * st + sa[u]];
                qj[u] = in[PJ * st + sa[u]];
                qm[u] = in[PM * st + sa[u]];
            }
        }
        for (int b = c0; b < c1; b += 32 * GG) {
            int src[GG];
            float px[GG], py[GG], pj[GG], pm[GG];
#pragma unroll
            for (int u = 0; u < GG; u++) {
                src[u] = sa[u];
                px[u] = qx[u];
                py[u] = qy[u];
                pj[u] = qj[u];
                pm[u] = qm[u];
                sa[u] = sb[u];
                if (sa[u] >= 0) {
                    qx[u] = in[PX * st + sa[u]];
                    qy[u] = in[PY * st + sa[u]];
                    qj[u] = in[PJ * st + sa[u]];
                    qm[u] = in[PM * st + sa[u]];
                }
            }
#pragma unroll
            for (int u = 0; u < GG; u++) sb[u] = src_at(b + 32 * (2 * GG + u) + lane);
#pragma unroll
            for (int u = 0; u < GG; u++) {
                const int slot = b + 32 * u + lane;
                int nkey = -1, ntile = -1;
                if (slot < c1) {
                    const Stencil2 sn = stencil2(px[u], py[u], nx, ny);
                    const int lx = sn.col - x0, ly = sn.row - y0;
                    Advected2 a;
                    if (lx >= 0 && lx < tx && ly >= 0 && ly < ty) {
                        const int wb = ly * wx + lx;
                        a = advect2(sn, px[u], py[u], pj[u], nx, ny, prm,
                                    [&](int o) { return vw[wb + (o / 3) * wx + o % 3]; }, [](int) { return 0.0f; });
                    } else {
                        set_status(B.status, ST_OOB);
                        const int sr = src[u];
                        a = Advected2{px[u], py[u], in[PU * st + sr], in[PV * st + sr], in[PC00 * st + sr],
                                      in[PC01 * st + sr], in[PC10 * st + sr], in[PC11 * st + sr], pj[u]};
                    }
                    out[PX * st + slot] = a.x;
                    out[PY * st + slot] = a.y;
                    out[PU * st + slot] = a.u;
                    out[PV * st + slot] = a.w;
                    out[PM * st + slot] = pm[u];
                    out[PJ * st + slot] = a.j;
                    out[PC00 * st + slot] = a.c00;
                    out[PC01 * st + slot] = a.c01;
                    out[PC10 * st + slot] = a.c10;
                    out[PC11 * st + slot] = a.c11;
                    batch_key(sc, a.x, a.y, nkey, ntile);
                    B.key[slot] = nkey;
                }
                warp_tally(B.cell_count, nkey, nkey >= 0, B.ncells, B.status);
                warp_tally(B.tile_count, ntile, ntile >= 0, B.nentries, B.status);
            }
        }
        __syncwarp();   // the window is free for the next chunk
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(B.done, 1u) == gridDim.x - 1) {   // the last CTA: the launch's end
            atomicExch(B.done, 0u);
            const unsigned long long start = *(volatile unsigned long long*)&B.phase_ns[NPHASE + 1];
            atomicAdd(&B.phase_ns[NPHASE - 1], global_ns() - start);
            atomicAdd(&B.phase_ns[NPHASE], 1ull);
        }
    }
}

// After a load: every particle's first cell key, tallied (the step's first phase expects the counts).
__global__ void __launch_bounds__(256) k_batch2_tally(Batch2 B) {
    const int n32 = (B.np + 31) & ~31;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n32; i += gridDim.x * blockDim.x) {
        int key = -1, tile = -1;
        if (i < B.np) {
            int lo = 0, hi = B.nscenes - 1;   // the scene owning slot i: the last with p0 <= i
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (B.scene[mid].p0 <= i) lo = mid;
                else hi = mid - 1;
            }
            const Scene2 sc = B.scene[lo];
            batch_key(sc, B.part[0][PX * B.stride + i], B.part[0][PY * B.stride + i], key, tile);
            B.key[i] = key;
        }
        warp_tally(B.cell_count, key, key >= 0, B.ncells, B.status);
        warp_tally(B.tile_count, tile, tile >= 0, B.nentries, B.status);
    }
}

// Grid readback: one float of every node of one scene.
__global__ void k_batch2_unpack(const float4* grid, float* out, int64_t nodes, int comp) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nodes) return;
    const float4 g = grid[i];
    out[i] = comp == 0 ? g.x : comp == 1 ? g.y : g.z;
}

const int TILES[][2] = VF_BATCH_TILES;
const int BLOCKS[] = VF_BATCH_BLOCKS;
constexpr int GRAPH_STEPS = 16;   // launches per graph replay

bool tile_ok(int tx, int ty) {
    for (auto& t : TILES)
        if (t[0] == tx && t[1] == ty) return true;
    return false;
}

bool block_ok(int b) {
    for (int x : BLOCKS)
        if (x == b) return true;
    return false;
}

}  // namespace

// ------------------------------------------------------------------ the handle

struct vf_mpm2_batch {
    std::vector<Scene2> scenes;
    uint32_t flags = 0;
    int block = 256, ctas = 0;
    size_t smem = 0;
    int64_t np = 0, stride = 0;
    int ncells = 0, nentries = 0;
    cudaStream_t stream = nullptr;
    DeviceBuffer scene_d, tile_scene, part[2], key, perm, cell_count, cursor, tile_count, tile_start[2], grid[2];
    DeviceBuffer chunk_start, scene_chunks, scene_chunk_start, item;
    DeviceBuffer ctl;      // step counter, two work counters, the done count, the barrier, the phase clock
    DeviceBuffer status;
    int64_t nodes = 0;
    int wmax = 0;
    int64_t steps = 0, launches = 0;
    bool loaded = false;
    bool timed_out = false;   // a grid barrier gave up: no step runs again until the next load
    cudaGraphExec_t graph = nullptr;
};

namespace {

Batch2 view(vf_mpm2_batch* h) {
    Batch2 b;
    b.scene = h->scene_d.as<Scene2>();
    b.nscenes = (int)h->scenes.size();
    b.tile_scene = h->tile_scene.as<int>();
    b.nentries = h->nentries;
    b.part[0] = h->part[0].as<float>();
    b.part[1] = h->part[1].as<float>();
    b.stride = h->stride;
    b.np = (int)h->np;
    b.ncells = h->ncells;
    b.key = h->key.as<int>();
    b.perm = h->perm.as<int>();
    b.cell_count = h->cell_count.as<int>();
    b.cursor = h->cursor.as<int>();
    b.tile_count = h->tile_count.as<int>();
    b.tile_start[0] = h->tile_start[0].as<int>();
    b.tile_start[1] = h->tile_start[1].as<int>();
    b.chunk_start = h->chunk_start.as<int>();
    b.scene_chunks = h->scene_chunks.as<int>();
    b.scene_chunk_start = h->scene_chunk_start.as<int>();
    b.item = h->item.as<int4>();
    b.item_cap = (int)(h->item.bytes / sizeof(int4));
    b.grid[0] = h->grid[0].as<float4>();
    b.grid[1] = h->grid[1].as<float4>();
    unsigned* ctl = h->ctl.as<unsigned>();
    b.step = ctl;
    b.work = ctl + 1;
    b.wmax = h->wmax;
    b.done = ctl + 3;
    b.bar = reinterpret_cast<GridBarrier*>(ctl + 4);
    b.phase_ns = reinterpret_cast<unsigned long long*>(ctl + 8);
    b.status = h->status.as<uint32_t>();
    return b;
}

int32_t launch_step(vf_mpm2_batch* h) {
    Batch2 b = view(h);
    void* args[] = {&b};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(h->ctas);
    cfg.blockDim = dim3(h->block);
    cfg.dynamicSmemBytes = h->smem;
    cfg.stream = h->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    VF_TRY_CUDA(cudaLaunchKernelExC(&cfg, (const void*)k_batch2_step, args));
    h->launches++;
    return VF_OK;
}

int32_t batch_status(vf_mpm2_batch* h) {
    uint32_t st = 0;
    VF_TRY_CUDA(cudaMemcpyAsync(&st, h->status.ptr, 4, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    if (st) {
        VF_TRY_CUDA(cudaMemsetAsync(h->status.ptr, 0, 4, h->stream));
        if (st & ST_TIMEOUT) h->timed_out = true;
        set_error("a batch kernel flagged device status 0x%x%s", st,
                  (st & ST_TIMEOUT) ? " (a grid barrier timed out; load the batch again before stepping it)" : "");
        return (st & ST_TIMEOUT) ? VF_ETIMEOUT : VF_EDEVICE;
    }
    return VF_OK;
}

// Captures GRAPH_STEPS step launches into one graph.
int32_t build_graph(vf_mpm2_batch* h) {
    if (h->graph) return VF_OK;
    cudaGraph_t g = nullptr;
    VF_TRY_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int32_t rc = VF_OK;
    for (int k = 0; k < GRAPH_STEPS && rc == VF_OK; k++) rc = launch_step(h);
    h->launches -= GRAPH_STEPS;   // captured, not run
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) {
        set_error("capturing the batch step failed: %s", cudaGetErrorString(e));
        return VF_ECUDA;
    }
    e = cudaGraphInstantiate(&h->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        h->graph = nullptr;
        set_error("instantiating the batch step graph failed: %s", cudaGetErrorString(e));
        return VF_ECUDA;
    }
    return VF_OK;
}

int32_t params_of(const vf_scene2& s, uint32_t flags, Params2* p) {
    float w[5];
    for (int k = 0; k < 5; k++) w[k] = bits_to_float(s.params[k]);
    VF_REQUIRE(w[0] > 0 && w[3] >= 0 && w[4] > 0, VF_EINVAL,   // Flip.java:204-207
               "dt > 0, bulk >= 0 and rho0 > 0, got dt %g, bulk %g, rho0 %g", w[0], w[3], w[4]);
    *p = Params2{w[0], w[1], w[2], w[3], w[4], (flags & VF_EOS_TAIT) ? 1 : 0,
                 (int)((flags & VF_WALL_STICKY_MASK) >> VF_WALL_STICKY_SHIFT)};
    return VF_OK;
}

}  // namespace

extern "C" {

int32_t vf_mpm2_batch_create(const vf_scene2* scenes, int32_t nscenes, uint32_t flags, int32_t block,
                             vf_mpm2_batch** out) {
    VF_REQUIRE(out, VF_EINVAL, "out is null");
    *out = nullptr;
    VF_REQUIRE(scenes && nscenes >= 1, VF_EINVAL, "a batch needs scenes, got %d", nscenes);
    VF_REQUIRE(!(flags & (VF_RELAX | VF_TENSION)), VF_EINVAL, "a batch steps plain scenes: no relaxation or tension");
    if (block == 0) block = 256;
    VF_REQUIRE(block_ok(block), VF_EINVAL, "block %d is not one of VF_BATCH_BLOCKS", block);
    std::vector<Scene2> sc((size_t)nscenes);
    int64_t np = 0, cells = 0, nodes = 0, entries = 0;
    int wmax = 0;
    for (int s = 0; s < nscenes; s++) {
        const vf_scene2& d = scenes[s];
        VF_REQUIRE(d.nx >= 3 && d.ny >= 3, VF_EINVAL, "scene %d: a grid needs at least three nodes each way, got %d x %d",
                   s, d.nx, d.ny);
        VF_REQUIRE(d.particles >= 1, VF_EINVAL, "scene %d: a step needs particles, got %d", s, d.particles);
        int tx = d.tile_x, ty = d.tile_y;
        if (tx == 0 && ty == 0) tx = ty = 16;
        VF_REQUIRE(tile_ok(tx, ty), VF_EINVAL, "scene %d: tile %d x %d is not one of VF_BATCH_TILES", s, tx, ty);
        Scene2& c = sc[s];
        int32_t rc = params_of(d, flags, &c.prm);
        if (rc) {
            set_error("scene %d: %s", s, last_error());
            return rc;
        }
        c.nx = d.nx;
        c.ny = d.ny;
        c.np = d.particles;
        c.tx = tx;
        c.ty = ty;
        c.ntx = (d.nx - 2 + tx - 1) / tx;
        c.nty = (d.ny - 2 + ty - 1) / ty;
        c.tc = tx * ty;
        c.p0 = (int)np;
        c.g0 = nodes;
        np += d.particles;
        nodes += (int64_t)d.nx * d.ny;
        cells += (int64_t)c.ntx * c.nty * c.tc;
        entries += (int64_t)c.ntx * c.nty + 1;
        wmax = std::max(wmax, (tx + 2) * (ty + 2));
    }
    VF_REQUIRE(np < (1ll << 31) - 64 && cells < (1ll << 31) && entries < (1ll << 30), VF_EINVAL,
               "a batch holds fewer than 2^31 particles and cell keys, got %lld and %lld", (long long)np,
               (long long)cells);
    // tile entries and cell keys laid out densest scene first, so the work-stealing phases take the
    // heaviest tiles first
    std::vector<int> order((size_t)nscenes);
    for (int s = 0; s < nscenes; s++) order[s] = s;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return (double)sc[a].np / ((double)sc[a].nx * sc[a].ny) > (double)sc[b].np / ((double)sc[b].nx * sc[b].ny);
    });
    std::vector<int> tile_scene((size_t)entries, -1);
    int t0 = 0, c0 = 0;
    for (int s : order) {
        Scene2& c = sc[s];
        c.t0 = t0;
        c.c0 = c0;
        const int nt = c.ntx * c.nty;
        for (int i = 0; i < nt; i++) tile_scene[(size_t)t0 + i] = s;
        t0 += nt + 1;
        c0 += nt * c.tc;
    }
    int32_t rc = require_device();
    if (rc) return rc;
    vf_mpm2_batch* h = new vf_mpm2_batch();
    h->scenes = sc;
    h->flags = flags;
    h->block = block;
    h->np = np;
    h->stride = (np + 63) / 64 * 64;
    h->ncells = (int)cells;
    h->nentries = (int)entries;
    h->nodes = nodes;
    h->wmax = wmax;
    h->smem = (size_t)(block / 32) * warp_smem_floats(wmax) * sizeof(float);
    auto fail = [&](int32_t code) {
        vf_mpm2_batch_destroy(h);
        return code;
    };
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        set_error("cudaStreamCreate failed");
        return fail(VF_ECUDA);
    }
    if (h->smem > 48 * 1024 &&
        cudaFuncSetAttribute(k_batch2_step, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)h->smem) != cudaSuccess) {
        set_error("cannot give the batch step %zu bytes of shared memory", h->smem);
        return fail(VF_ECUDA);
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch2_step, block, h->smem) != cudaSuccess ||
        per_sm < 1) {
        set_error("the batch step does not fit on an SM with %d threads and %zu bytes of shared memory", block, h->smem);
        return fail(VF_ECUDA);
    }
    h->ctas = per_sm * sm_count();
    const size_t pb = (size_t)h->stride * NF2 * 4;
    if ((rc = h->scene_d.alloc(sc.size() * sizeof(Scene2))) || (rc = h->tile_scene.alloc((size_t)entries * 4)) ||
        (rc = h->part[0].alloc(pb)) || (rc = h->part[1].alloc(pb)) || (rc = h->key.alloc((size_t)np * 4)) ||
        (rc = h->perm.alloc((size_t)np * 4)) || (rc = h->cell_count.alloc((size_t)cells * 4)) ||
        (rc = h->cursor.alloc((size_t)cells * 4)) || (rc = h->tile_count.alloc((size_t)entries * 4)) ||
        (rc = h->tile_start[0].alloc((size_t)entries * 4)) || (rc = h->tile_start[1].alloc((size_t)entries * 4)) ||
        (rc = h->grid[0].alloc((size_t)nodes * 16)) || (rc = h->grid[1].alloc((size_t)nodes * 16)) ||
        (rc = h->chunk_start.alloc((size_t)entries * 4)) || (rc = h->scene_chunks.alloc((size_t)nscenes * 4)) ||
        (rc = h->scene_chunk_start.alloc((size_t)(nscenes + 1) * 4)) ||
        (rc = h->item.alloc((size_t)(np / CHUNK + entries + 1) * sizeof(int4))) ||
        (rc = h->ctl.alloc(128)) || (rc = h->status.alloc(16)))
        return fail(rc);
    if (cudaMemcpyAsync(h->scene_d.ptr, sc.data(), sc.size() * sizeof(Scene2), cudaMemcpyHostToDevice, h->stream) !=
            cudaSuccess ||
        cudaMemcpyAsync(h->tile_scene.ptr, tile_scene.data(), (size_t)entries * 4, cudaMemcpyHostToDevice, h->stream) !=
            cudaSuccess ||
        cudaMemsetAsync(h->status.ptr, 0, h->status.bytes, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess) {
        set_error("uploading the scene table failed");
        return fail(VF_ECUDA);
    }
    *out = h;
    return VF_OK;
}

int32_t vf_mpm2_batch_load(vf_mpm2_batch* h, const float* x, const float* y, const float* u, const float* v,
                           const float* m) {
    VF_REQUIRE(h && x && y && u && v && m, VF_EINVAL, "null argument");
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    float* base = h->part[0].as<float>();
    const float* src[5] = {x, y, u, v, m};
    for (int f = 0; f < 5; f++)
        VF_TRY_CUDA(cudaMemcpyAsync(base + f * h->stride, src[f], (size_t)h->np * 4, cudaMemcpyHostToDevice, h->stream));
    VF_TRY_CUDA(fill_f32(base + PJ * h->stride, h->np, 1.0f, h->stream));
    VF_TRY_CUDA(cudaMemsetAsync(base + PC00 * h->stride, 0, (size_t)4 * h->stride * 4, h->stream));
    for (DeviceBuffer* b : {&h->cell_count, &h->tile_count, &h->tile_start[0], &h->tile_start[1], &h->grid[0],
                            &h->grid[1], &h->ctl, &h->status})
        VF_TRY_CUDA(cudaMemsetAsync(b->ptr, 0, b->bytes, h->stream));
    Batch2 b = view(h);
    k_batch2_tally<<<std::max(1, std::min(div_up(h->np, 256), sm_count() * 8)), 256, 0, h->stream>>>(b);
    VF_CHECK_LAUNCH();
    h->launches++;
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    h->steps = 0;
    h->loaded = true;
    h->timed_out = false;
    return batch_status(h);
}

int32_t vf_mpm2_batch_advance(vf_mpm2_batch* h, int32_t count) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    VF_REQUIRE(count >= 0, VF_EINVAL, "count >= 0, got %d", count);
    VF_REQUIRE(h->loaded, VF_ESTATE, "load the batch before stepping it");
    VF_REQUIRE(!h->timed_out, VF_ESTATE, "a grid barrier of this batch timed out; load it again before stepping it");
    int32_t rc;
    int left = count;
    if (left >= GRAPH_STEPS) {
        if ((rc = build_graph(h))) return rc;
        for (; left >= GRAPH_STEPS; left -= GRAPH_STEPS) {
            VF_TRY_CUDA(cudaGraphLaunch(h->graph, h->stream));
            h->launches += GRAPH_STEPS;
        }
    }
    for (; left > 0; left--)
        if ((rc = launch_step(h))) return rc;
    h->steps += count;
    return VF_OK;
}

int32_t vf_mpm2_batch_set_wait_limit(vf_mpm2_batch* h, int32_t polls) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    VF_REQUIRE(polls >= 0, VF_EINVAL, "polls >= 0, got %d", polls);
    const unsigned v = (unsigned)polls;
    unsigned* limit = &reinterpret_cast<GridBarrier*>(h->ctl.as<unsigned>() + 4)->limit;
    VF_TRY_CUDA(cudaMemcpyAsync(limit, &v, 4, cudaMemcpyHostToDevice, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return VF_OK;
}

int32_t vf_mpm2_batch_finish(vf_mpm2_batch* h) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    return batch_status(h);
}

int32_t vf_mpm2_batch_read(vf_mpm2_batch* h, int32_t scene, int32_t field, float* out, int64_t n) {
    VF_REQUIRE(h && out, VF_EINVAL, "null argument");
    VF_REQUIRE(scene >= 0 && scene < (int)h->scenes.size(), VF_EINVAL, "no scene %d", scene);
    VF_REQUIRE(h->loaded, VF_ESTATE, "the batch holds no particles yet");
    const Scene2& sc = h->scenes[scene];
    int32_t rc = batch_status(h);
    if (rc) return rc;
    if (field >= VF2_X && field <= VF2_C11) {
        VF_REQUIRE(n == sc.np, VF_EINVAL, "scene %d holds %d particles, got %lld", scene, sc.np, (long long)n);
        const float* src = h->part[h->steps & 1].as<float>() + (int64_t)field * h->stride + sc.p0;
        VF_TRY_CUDA(cudaMemcpyAsync(out, src, (size_t)n * 4, cudaMemcpyDeviceToHost, h->stream));
    } else if (field >= VF2_GM && field <= VF2_GMV) {
        const int64_t nodes = (int64_t)sc.nx * sc.ny;
        VF_REQUIRE(n == nodes, VF_EINVAL, "scene %d has %lld nodes, got %lld", scene, (long long)nodes, (long long)n);
        VF_REQUIRE(h->steps > 0, VF_ESTATE, "no step has run");
        DeviceBuffer tmp;
        if ((rc = tmp.alloc((size_t)nodes * 4))) return rc;
        const float4* g = h->grid[(h->steps - 1) & 1].as<float4>() + sc.g0;
        k_batch2_unpack<<<div_up(nodes, 256), 256, 0, h->stream>>>(g, tmp.as<float>(), nodes, field - VF2_GM);
        VF_CHECK_LAUNCH();
        VF_TRY_CUDA(cudaMemcpyAsync(out, tmp.ptr, (size_t)nodes * 4, cudaMemcpyDeviceToHost, h->stream));
        VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    } else {
        set_error("no field %d", field);
        return VF_EINVAL;
    }
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return VF_OK;
}

int32_t vf_mpm2_batch_config(const vf_mpm2_batch* h, int32_t scene, int32_t* tile_x, int32_t* tile_y, int32_t* block,
                             int32_t* ctas) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    VF_REQUIRE(scene >= 0 && scene < (int)h->scenes.size(), VF_EINVAL, "no scene %d", scene);
    if (tile_x) *tile_x = h->scenes[scene].tx;
    if (tile_y) *tile_y = h->scenes[scene].ty;
    if (block) *block = h->block;
    if (ctas) *ctas = h->ctas;
    return VF_OK;
}

int32_t vf_mpm2_batch_phases(vf_mpm2_batch* h, double ms[5], int64_t* launches) {
    VF_REQUIRE(h && ms, VF_EINVAL, "null argument");
    unsigned long long ns[NPHASE + 1];
    unsigned long long* dev = reinterpret_cast<unsigned long long*>(h->ctl.as<unsigned>() + 8);
    VF_TRY_CUDA(cudaMemcpyAsync(ns, dev, sizeof ns, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    for (int k = 0; k < NPHASE; k++) ms[k] = (double)ns[k] / 1e6;
    if (launches) *launches = (int64_t)ns[NPHASE];
    VF_TRY_CUDA(cudaMemsetAsync(dev, 0, sizeof ns, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return VF_OK;
}

int64_t vf_mpm2_batch_particles(const vf_mpm2_batch* h) { return h ? h->np : 0; }
int64_t vf_mpm2_batch_steps(const vf_mpm2_batch* h) { return h ? h->steps : 0; }
int64_t vf_mpm2_batch_launches(const vf_mpm2_batch* h) { return h ? h->launches : 0; }
void* vf_mpm2_batch_stream(vf_mpm2_batch* h) { return h ? (void*)h->stream : nullptr; }

void vf_mpm2_batch_destroy(vf_mpm2_batch* h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->graph) cudaGraphExecDestroy(h->graph);
    for (DeviceBuffer* b : {&h->scene_d, &h->tile_scene, &h->part[0], &h->part[1], &h->key, &h->perm, &h->cell_count,
                            &h->cursor, &h->tile_count, &h->tile_start[0], &h->tile_start[1], &h->grid[0], &h->grid[1],
                            &h->chunk_start, &h->scene_chunks, &h->scene_chunk_start, &h->item, &h->ctl,
                            &h->status})
        b->release();
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

}  // extern "C"
