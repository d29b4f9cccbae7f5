// mpm3_kernels.cuh -- the 3D MLS-MPM/APIC step's kernels (Flip3.java), for sm_100a.
//
// Layout in HBM:
//   particles  two buffer sets (ping-pong), each 17 SoA f32 fields of `stride` floats:
//              x y z u v w m j c00 c01 c02 c10 c11 c12 c20 c21 c22   (Flip3.PARTICLE order)
//   grid       float4 per node {m, mu, mv, mw}, node (k*ny + j)*nx + i, two buffers (one per step
//              parity, so the last scatter stays readable while the next one accumulates)
//   velocity   float4 per node {u, v, w, 0} (dense pipeline, and any step with surface tension; otherwise the
//              tiled G2P computes the grid update into shared memory and never writes velocities to HBM)
//   tension    two colour planes and six stress planes of nodes floats, when the step has surface tension
//   sort       key/perm per particle; cell counts/starts/cursors over the brick-major keys; brick
//              counts/starts and the list of non-empty bricks
#pragma once

#include "common.cuh"
#include "sort.cuh"

namespace vf {

enum Field3 { X = 0, Y, Z, U, V, W, M, J, C00, C01, C02, C10, C11, C12, C20, C21, C22, NF3 };

struct Dims3 {
    int nx, ny, nz;
    int nbx, nby, nbz;   // bricks of 8^3 stencil cells per axis
};

// Device copy of Flip3.params (Flip3.java:55-64) plus the physics options.
struct Params3 {
    float dt, gx, gy, gz, bulk, rho0, sigma;
    int tait;     // VF_EOS_TAIT
    int sticky;   // wall thickness in nodes; 0 = the reference's wall ring
};

constexpr float EMPTY3 = 1e-9f;    // Flip3.java:71
constexpr float J_BOUND3 = 10.0f;  // Flip3.java:74
constexpr int BRICK = 8;
constexpr int WIN = BRICK + 2;                 // nodes per axis a brick's particles reach
constexpr int WIN3 = WIN * WIN * WIN;          // 1000

// Stencil3.of (Flip3.java:664-679): cell in [0, n-3], offset in [1/2, 3/2].
__device__ __forceinline__ void stencil_axis(float at, int size, int& cell, float& off) {
    float x = clampf(at, 0.5f, (float)size - 1.5f);
    cell = (int)fminf(__fsub_rn(x, 0.5f), (float)(size - 3));
    off = __fsub_rn(x, (float)cell);
}

// The brick-major key of a stencil cell (see oracle/mpm3.c or_key3).
__device__ __forceinline__ int key3_of_cell(int cx, int cy, int cz, const Dims3& d) {
    int brick = ((cz >> 3) * d.nby + (cy >> 3)) * d.nbx + (cx >> 3);
    int local = ((cz & 7) * 8 + (cy & 7)) * 8 + (cx & 7);
    return brick * 512 + local;
}

__device__ __forceinline__ int key3_of(float x, float y, float z, const Dims3& d) {
    int c[3];
    float o;
    stencil_axis(x, d.nx, c[0], o);
    stencil_axis(y, d.ny, c[1], o);
    stencil_axis(z, d.nz, c[2], o);
    return key3_of_cell(c[0], c[1], c[2], d);
}

// The grid update of one node (Flip3.grid, Flip3.java:267-311): momentum over mass plus a step of
// gravity, zero for an empty node; the wall ring drops the velocity into the wall, or a sticky
// wall of `sticky` nodes stops it.
// Flip3.grid's velocity before the walls (Flip3.java:285-290): momentum over mass plus a step of gravity.
__device__ __forceinline__ void grid_velocity_free(float4 g, const Params3& p, float v[3]) {
    v[0] = v[1] = v[2] = 0.0f;
    const float mass = g.x;
    if (mass > EMPTY3) {
        v[0] = __fadd_rn(__fdiv_rn(g.y, mass), __fmul_rn(p.dt, p.gx));
        v[1] = __fadd_rn(__fdiv_rn(g.z, mass), __fmul_rn(p.dt, p.gy));
        v[2] = __fadd_rn(__fdiv_rn(g.w, mass), __fmul_rn(p.dt, p.gz));
    }
}

// Flip3.grid's walls (Flip3.java:302-307): the velocity into the wall ring dropped, or with sticky walls every
// node within `sticky` of an edge stopped.
__device__ __forceinline__ float3 grid_walls(float v[3], int i, int j, int k, const Dims3& d, const Params3& p) {
    const int at[3] = {i, j, k};
    const int size[3] = {d.nx, d.ny, d.nz};
    if (p.sticky > 0) {
        bool stuck = false;
#pragma unroll
        for (int a = 0; a < 3; a++) stuck |= at[a] < p.sticky || at[a] > size[a] - 1 - p.sticky;
        if (stuck) v[0] = v[1] = v[2] = 0.0f;
    } else {
#pragma unroll
        for (int a = 0; a < 3; a++) {
            if (!(at[a] > 1)) v[a] = fmaxf(v[a], 0.0f);
            if (at[a] > size[a] - 3) v[a] = fminf(v[a], 0.0f);
        }
    }
    return make_float3(v[0], v[1], v[2]);
}

__device__ __forceinline__ float3 grid_velocity(float4 g, int i, int j, int k, const Dims3& d, const Params3& p) {
    float v[3];
    grid_velocity_free(g, p, v);
    return grid_walls(v, i, j, k, d, p);
}

// Flip3.keepInside (Flip3.java:644-655)
__device__ __forceinline__ void keep_inside(float& at, float& vel, int size) {
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

// Kernel parameter bundle.
struct Step3 {
    const float* in;        // current particle set
    float* out;             // next particle set (== in when not sorting)
    int64_t stride;         // floats per field
    int np;
    int* perm;              // sorted slot -> source particle, or null (identity, in place); the tiled
                            // scatter puts each cell's run in ascending order in place
    float4* grid;           // this step's grid {m, mu, mv, mw}
    float4* vel;            // dense pipeline's node velocities
    const Params3* params;
    Dims3 d;
    uint32_t* status;
    // sort bookkeeping
    int* key;               // per particle (indexed by slot in `out`)
    int* cell_count;
    int* brick_count;
    const int* cell_start;
    const int* brick_start;
    const int* active;
    const int* n_active;
    int* work;              // the tiled G2P's item counter (zeroed by the brick scan that made `active`)
    int64_t nkeys;
    int nbricks;
    int count_next;         // G2P also counts keys for the next step's sort
    int vel_ready;          // the tiled G2P reads `vel` (written by the grid pass) instead of updating the grid itself
    int g2p_split;          // the tiled G2P's work items per brick (>= 1): each loads the brick's window and takes
                            // one slice of its particles, so a scene of few bricks still fills the GPU
    // sparse node storage: the grid is a pool of POOL_BRICK^3-node bricks, `page` maps each brick position of the
    // domain (pnx x pny x pnz, x fastest) to its slot in the pool, or -1
    int sparse;
    const int* page;
    int pool_cap;           // slots in the pool
    int pnx, pny, pnz;
};

constexpr int POOL_BRICK = 8;
constexpr int POOL_NODES = POOL_BRICK * POOL_BRICK * POOL_BRICK;   // 512 nodes, 8 KB of float4 a brick

// The address of node (gx, gy, gz) in this step's grid: the dense box, or the node's brick's slot in the pool,
// nodes x fastest within a brick. Null for a brick with no slot (the pool overflowed).
__device__ __forceinline__ float4* node_addr(const Step3& s, int gx, int gy, int gz) {
    if (!s.sparse) return s.grid + ((int64_t)gz * s.d.ny + gy) * s.d.nx + gx;
    const int slot = s.page[((gz >> 3) * s.pny + (gy >> 3)) * s.pnx + (gx >> 3)];
    if ((unsigned)slot >= (unsigned)s.pool_cap) return nullptr;
    return s.grid + (int64_t)slot * POOL_NODES + (((gz & 7) * POOL_BRICK + (gy & 7)) * POOL_BRICK + (gx & 7));
}

// The exact (fixed-point) scatter: each node amount of Flip3.scatter in the reference's operand order without
// FMA contraction, quantized to FIXED3_BITS fractional bits (round to nearest even) and added with 64-bit
// integer atomics into q[4][nodes] (m, mu, mv, mw), so the sums do not depend on the order of the additions.
// A particle's 27 mass shares are quantized and the centre node takes the rest of its quantized mass, so the
// grid's total mass is the particles' quantized masses' sum exactly.
constexpr int FIXED3_BITS = 40;
__global__ void k_p2g3_fixed(Step3 s, unsigned long long* q);
// q (FIXED3_BITS fractional bits) -> the float grid: float(double(q) * 2^-FIXED3_BITS) per component.
__global__ void k_fixed_to_grid3(const long long* q, float4* grid, int64_t nodes);

// Surface tension (Tension3.java), the passes between the scatter and the grid when a step has tension:
//   blur    x TENSION3_BLURS: the [1 2 1]^3/64 blur of the node mass taken to a colour (first pass) or of the
//           last colour, every read held to the wall ring; one thread per node
//   stress  the capillary stress over sigma from the colour's central differences, six planes of nodes
//           (txx tyy tzz txy txz tyz)
//   grid    k_grid3_tension: Flip3.grid plus dt sigma F / max(m, MASS_FLOOR rho0), F the stress's flux across
//           the node's open faces; writes `vel` for the G2P
constexpr int TENSION3_BLURS = 6;          // Flip.TENSION_BLURS
// One blur: scaled (the first, src = the grid's float4 {m, ...}) or of the last colour (src = float[nodes]).
cudaError_t launch_tension3_blur(bool scaled, const void* src, float* dst, const Params3* params, const Dims3& d,
                                 cudaStream_t stream);
cudaError_t launch_tension3_stress(const float* colour, float* stress, const Dims3& d, cudaStream_t stream);
__global__ void k_grid3_tension(Step3 s, const float* colour, const float* stress);

// Sparse node storage (a page table of 8^3-node bricks over one pool). Each step that scatters rebuilds the
// page of the grid buffer it scatters into from that step's non-empty cell bricks: a cell brick's 10^3 node
// window covers its own node brick and the next one along each axis, so those 8 are marked, and the marked
// bricks take slots 0.. in brick order. The grid holds nothing from one step to the next, so no slot is kept.
__global__ void k_pool_mark3(Step3 s, int* mark);
__global__ void k_pool_page3(int* mark, int* page, int npages, int* n_used, int cap, uint32_t* status);
__global__ void k_pool_clear3(float4* pool, const int* n_used);
// The pool through its page as a dense grid (zero where no brick is), for readouts.
__global__ void k_pool_unpack3(Step3 s, float4* dense);

__global__ void k_key_count3(Step3 s);
__global__ void k_p2g3_atomic(Step3 s);
__global__ void k_p2g3_warp(Step3 s);
// The tiled scatter (work units of 8x8x1 cells): 128 threads a CTA, two CTAs an SM.
cudaError_t launch_p2g3_tile(int blocks, const Step3& s, cudaStream_t stream);
// The fused step (mpm3_fused.cu): the gather from s.grid of the particles sorted by s.perm, written to their slots
// in s.out, and their scatter into grid_out; 256 threads a CTA, two CTAs an SM, one CTA per half brick.
cudaError_t launch_g2p2g3(int blocks, const Step3& s, float4* grid_out, cudaStream_t stream);
cudaError_t fused_prepare();    // its shared-memory attribute
int fused_blocks_per_sm();      // the CTAs an SM holds
size_t p2g_tile_smem();
cudaError_t p2g_tile_prepare();   // its shared-memory attribute
__global__ void k_grid3_dense(Step3 s);
__global__ void k_g2p3(Step3 s);
__global__ void k_g2p3_tile(Step3 s);
__global__ void k_clear_bricks3(Step3 s);
__global__ void k_touched3(const float4* grid, int64_t nodes, unsigned long long* out);
// The smallest positive mass as float bits into *out (which starts at FLT_MAX's bits): positive floats order as
// their bits do, so an integer atomicMin finds it.
__global__ void k_min_positive3(const float* m, int n, unsigned* out);
__global__ void k_unpack_grid3(const float4* grid, float* out, int64_t nodes, int comp);

// ParticleDiagnostics.of's order statistics of a device J (pdiag.cu): out = {valid count, min bits, max bits,
// bits at the 99th percentile rank, bits at the 1st}; scratch of pdiag_scratch_bytes().
size_t pdiag_scratch_bytes();
int32_t pdiag_run(const float* j, int64_t n, void* scratch, cudaStream_t s, unsigned out[5]);

}  // namespace vf
