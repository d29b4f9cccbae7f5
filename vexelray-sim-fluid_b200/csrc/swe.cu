// swe.cu -- the shallow-water step (ShallowWater.java) on TMA-staged shared-memory halo tiles,
// and the vf_swe_* C-ABI: PatchSimulation (vexelray-sim-fluid-gui/.../gui/PatchSimulation.java).
// Reference paths: vexelray-sim-fluid-core/src/main/java/dev/vexelray/sim/fluid/stencil/.
//
// Built with --fmad=false and IEEE division and square root: every operation rounds as the
// reference's strict f32 (Java) arithmetic does, so a step's output is bit-identical to the
// reference's CPU semantics (and to the oracle), and so are the tick counts it derives.
//
// A second arithmetic, the fast mode (vf_swe_set_exact(h, 0)), keeps the flux form but rounds differently:
// fused multiply-adds (written out as fmaf, since the file forbids contraction), one approximate reciprocal of a
// cell's depth shared by its two velocities, one approximate reciprocal of each face's wave span shared by its
// three fluxes, and an approximate square root for the wave speed; and it runs as a column walk in registers over
// a TMA-staged tile (k_swe_strip<false>) instead of staging primitives and fluxes in shared memory. It is within a
// stated tolerance of the reference rather than equal to it, and the water still moves only between neighbours.
// The tick count from the previous step's speed stays IEEE. The exact mode can walk strips too
// (vf_swe_set_tile_width(h, 0), k_swe_strip<true>): bit-identical, and measured slower than the tile below.
//
// One CTA per 64 x 16 tile of cells (k_swe_tile):
//   1. the tile and a one-cell halo of h, hu, hv land in shared memory by three 2D TMA loads
//      (the box starts four cells left of the tile so its x coordinate is 16-byte aligned);
//   2. per cell of tile+halo: u = hu/h, v = hv/h (0 when dry) and c = sqrt(g h), once;
//   3. every x-face and y-face flux of the tile computed ONCE (the reference computes each face
//      twice, once from each side, with identical inputs and so identical bits);
//   4. each cell's update from its four faces, the depth clamp (counted), the stores, and the next
//      step's speed max-reduced over the CTA before one filtered atomicMax.
#include <cuda.h>

#include <cmath>
#include <vector>

#include "profiler.cuh"
#include "snapshot.cuh"
#include "sort.cuh"

using namespace vf;

namespace {

// A tile is TX x 16 cells, TX = 64 (the default) or 32 (vf_swe_set_tile_width).
template <int TX_>
struct Tile {
    static constexpr int TX = TX_, TY = 16;
    static constexpr int HX = TX + 8;                  // loaded box width: x0-4 .. x0+TX+3
    static constexpr int HY = TY + 2;                  // loaded box height: y0-1 .. y0+TY
    static constexpr int PX = TX + 2, PY = TY + 2;     // primitive window: x0-1 .. x0+TX
    static constexpr int BOXF = (HY * HX * 4 + 127) / 128 * 128 / 4;   // floats per staged field, 128-byte padded
};
constexpr int SWE_THREADS = 256;
constexpr int SWE_TY = 16;

struct SweArgs {
    const float* in[3];
    float* out[3];
    const float* params;                        // [g, courant, dx, dy, dry] (ShallowWater.java:120)
    const int* speed_in;
    int* speed_out;
    int* speed_clear;
    const int* budget_in;
    int* budget_out;
    int* clamped;
    uint32_t* status;
    int nx, ny;
    int edge[4];                                // west, east, south, north: VF_EDGE_*
    int use_tma;
};

template <int TX_>
struct SweShared {
    using T = Tile<TX_>;
    float box[3][T::BOXF];                                    // h, hu, hv, each [HY][HX] (TMA destinations)
    float pu[T::PY][T::PX], pv[T::PY][T::PX], pc[T::PY][T::PX];   // primitives
    float fx[3][T::TY][T::TX + 1];                            // x-face fluxes (mass, normal=hu, tangent=hv)
    float fy[3][T::TY + 1][T::TX];                            // y-face fluxes (mass, normal=hv, tangent=hu)
    unsigned long long bar;
    int red[SWE_THREADS / 32];
    int clamps;
};

struct Face {
    float mass, normal, tangent;
};

// ShallowWater.hll (ShallowWater.java:336-378) with the side's velocities and wave speed given.
__device__ __forceinline__ Face hll(float g, float dry, float hL, float qnL, float qtL, float unL, float utL, float cL,
                                    float hR, float qnR, float qtR, float unR, float utR, float cR) {
    float sL = fminf(unL - cL, unR - cR);
    float sR = fmaxf(unL + cL, unR + cR);
    if (!(hR > dry)) {
        sL = unL - cL;
        sR = unL + 2.0f * cL;
    }
    if (!(hL > dry)) {
        sL = unR - 2.0f * cR;
        sR = unR + cR;
    }
    const float lo = fminf(sL, 0.0f);
    const float hi = fmaxf(sR, 0.0f);
    const float span = fmaxf(hi - lo, 1e-30f);
    const float lohi = lo * hi;
    const float pL = (0.5f * g) * (hL * hL);
    const float pR = (0.5f * g) * (hR * hR);
    Face f;
    // ShallowWater.combine (381-384): ((hi FL - lo FR) + lo hi (UR - UL)) / span
    f.mass = ((hi * qnL - lo * qnR) + lohi * (hR - hL)) / span;
    f.normal = ((hi * (qnL * unL + pL) - lo * (qnR * unR + pR)) + lohi * (qnR - qnL)) / span;
    f.tangent = ((hi * (qnL * utL) - lo * (qnR * utR)) + lohi * (qtR - qtL)) / span;
    return f;
}

__device__ __forceinline__ float velocity(float h, float q, float dry) { return h > dry ? q / h : 0.0f; }

// The fast mode's HLL: the same wave speeds and flux form as hll(), the division by the span done once as an
// approximate reciprocal and the products fused; two faces at once, one in each half of paired fp32
// (FFMA2/FADD2/FMUL2): the column walk's x-face and y-face of a row, which are independent.
struct Face2 {
    float2 mass, normal, tangent;
};

__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 min2(float2 a, float2 b) { return make_float2(fminf(a.x, b.x), fminf(a.y, b.y)); }
__device__ __forceinline__ float2 max2(float2 a, float2 b) { return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }

__device__ __forceinline__ Face2 hll_fast2(float g, float dry, float2 hL, float2 qnL, float2 qtL, float2 unL, float2 utL,
                                           float2 cL, float2 hR, float2 qnR, float2 qtR, float2 unR, float2 utR,
                                           float2 cR) {
    const float2 lm = __fadd2_rn(unL, neg2(cL)), lp = __fadd2_rn(unL, cL);
    const float2 rm = __fadd2_rn(unR, neg2(cR)), rp = __fadd2_rn(unR, cR);
    float2 sL = min2(lm, rm), sR = max2(lp, rp);
    const float2 two = f2(2.0f, 2.0f);
    const float2 l2 = __ffma2_rn(two, cL, unL), r2 = __ffma2_rn(neg2(two), cR, unR);
    if (!(hR.x > dry)) { sL.x = lm.x; sR.x = l2.x; }
    if (!(hR.y > dry)) { sL.y = lm.y; sR.y = l2.y; }
    if (!(hL.x > dry)) { sL.x = r2.x; sR.x = rp.x; }
    if (!(hL.y > dry)) { sL.y = r2.y; sR.y = rp.y; }
    const float2 zero = f2(0.0f, 0.0f);
    const float2 lo = min2(sL, zero), hi = max2(sR, zero);
    const float2 span = max2(__fadd2_rn(hi, neg2(lo)), f2(1e-30f, 1e-30f));
    const float2 inv = f2(__fdividef(1.0f, span.x), __fdividef(1.0f, span.y));
    const float2 lohi = __fmul2_rn(lo, hi);
    const float2 hg = f2(0.5f * g, 0.5f * g);
    const float2 pL = __fmul2_rn(hg, __fmul2_rn(hL, hL)), pR = __fmul2_rn(hg, __fmul2_rn(hR, hR));
    const float2 loqR = __fmul2_rn(lo, qnR), hiqL = __fmul2_rn(hi, qnL);
    Face2 f;
    f.mass = __fmul2_rn(__ffma2_rn(lohi, __fadd2_rn(hR, neg2(hL)), __fadd2_rn(hiqL, neg2(loqR))), inv);
    const float2 fl = __ffma2_rn(qnL, unL, pL), fr = __ffma2_rn(qnR, unR, pR);
    f.normal = __fmul2_rn(__ffma2_rn(lohi, __fadd2_rn(qnR, neg2(qnL)), __ffma2_rn(hi, fl, neg2(__fmul2_rn(lo, fr)))), inv);
    f.tangent =
        __fmul2_rn(__ffma2_rn(lohi, __fadd2_rn(qtR, neg2(qtL)), __ffma2_rn(hiqL, utL, neg2(__fmul2_rn(loqR, utR)))), inv);
    return f;
}

// The fast mode's square root (approximate reciprocal square root; zero at zero).
__device__ __forceinline__ float sqrt_fast(float x) { return x > 0.0f ? x * rsqrtf(x) : 0.0f; }

__device__ __forceinline__ bool poll_barrier(uint32_t addr, int phase, int limit) {
    for (int it = 0; it < limit; it++) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(addr), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Bounded wait on an mbarrier phase. On giving up it sets the status bit, then waits once more,
// again bounded, so copies still in flight land before the CTA leaves; returns false.
__device__ __forceinline__ bool wait_barrier(unsigned long long* bar, int phase, uint32_t* status) {
    const uint32_t addr = (uint32_t)__cvta_generic_to_shared(bar);
    if (poll_barrier(addr, phase, 1 << 22)) return true;
    set_status(status, ST_TIMEOUT);
    poll_barrier(addr, phase, 1 << 22);
    return false;
}

// One tile (tx, ty) of one step. The CTA's mbarrier is initialised; `parity` is the phase its TMA completes.
// Returns false (status set, nothing written) when the TMA did not land within the bounded wait.
template <int TX_>
__device__ __forceinline__ bool swe_tile(const SweArgs& a, const CUtensorMap* tm_h, const CUtensorMap* tm_hu,
                                         const CUtensorMap* tm_hv, SweShared<TX_>& S, int tx, int ty, int parity) {
    using T = Tile<TX_>;
    constexpr int TX = T::TX, TY = T::TY, HX = T::HX, HY = T::HY, PX = T::PX, PY = T::PY;
    const int tid = threadIdx.x;
    const int x0 = tx * TX, y0 = ty * TY;
    const int nx = a.nx, ny = a.ny;

    // ShallowWater.java:184-192: the step from the fastest wave, in whole ticks, within the budget
    const float g = a.params[0], courant = a.params[1], dx = a.params[2], dy = a.params[3], dry = a.params[4];
    const float fastest = __int_as_float(__ldcg(a.speed_in));
    const float allowed = fminf((courant * fminf(dx, dy)) / fmaxf(fastest, 1e-30f), 2000.0f);
    int ticks = (int)(allowed * 1000000.0f);
    const int budget = __ldcg(a.budget_in);
    if (budget < ticks) ticks = budget;
    const float dt = (float)ticks * (float)(1.0 / 1000000.0);
    const float rx = dt / dx;
    const float ry = dt / dy;

    // 1. stage the tile + halo
    bool loaded = true;
    if (tid == 0) S.clamps = 0;
    if (a.use_tma) {
        if (tid == 0) {
            // the previous tile's reads of the box (generic proxy) before this tile's TMA writes (async proxy)
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&S.bar);
            const uint32_t bytes = 3u * HY * HX * 4u;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
            const CUtensorMap* maps[3] = {tm_h, tm_hu, tm_hv};
            const int bx = x0 - 4, by = y0 - 1;   // bx is a multiple of 4: 16-byte aligned
            for (int f = 0; f < 3; f++) {
                const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&S.box[f][0]);
                asm volatile(
                    "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
                    "[%4];" ::"r"(dst),
                    "l"(maps[f]), "r"(bx), "r"(by), "r"(bar)
                    : "memory");
            }
        }
        loaded = wait_barrier(&S.bar, parity, a.status);
    } else {
        for (int i = tid; i < HY * HX; i += SWE_THREADS) {
            const int ly = i / HX, lx = i % HX;
            const int gx = x0 - 4 + lx, gy = y0 - 1 + ly;
            const bool in = gx >= 0 && gx < nx && gy >= 0 && gy < ny;
            const int64_t c = (int64_t)gy * nx + gx;
            for (int f = 0; f < 3; f++) S.box[f][ly * HX + lx] = in ? __ldcg(a.in[f] + c) : 0.0f;
        }
    }
    // a TMA that never landed: the status word says so, nothing of the tile is written
    if (!__syncthreads_and(loaded)) return false;

    // 2. primitives of tile + halo (cells x0-1..x0+TX, y0-1..y0+TY that lie in the domain)
    for (int i = tid; i < PY * PX; i += SWE_THREADS) {
        const int ly = i / PX, lx = i % PX;
        const float h = S.box[0][(ly) * HX + lx + 3];
        S.pu[ly][lx] = velocity(h, S.box[1][(ly) * HX + lx + 3], dry);
        S.pv[ly][lx] = velocity(h, S.box[2][(ly) * HX + lx + 3], dry);
        S.pc[ly][lx] = sqrtf(g * h);
    }
    __syncthreads();

    // 3a. x-faces: face fx is the west face of cell fx (left = fx-1, right = fx)
    for (int i = tid; i < TY * (TX + 1); i += SWE_THREADS) {
        const int ly = i / (TX + 1), lf = i % (TX + 1);
        const int gy = y0 + ly, gf = x0 + lf;
        if (gy >= ny || gf > nx) continue;
        // local primitive/box column of the left cell is lf (box: lf + 3)
        int l = lf, r = lf + 1;       // primitive columns of left and right cells
        float sgnL = 1.0f, sgnR = 1.0f;
        if (gf == 0) {                // left is the ghost of cell 0
            l = r;
            if (a.edge[0] == VF_EDGE_WALL) sgnL = -1.0f;
        }
        if (gf == nx) {               // right is the ghost of cell nx-1
            r = l;
            if (a.edge[1] == VF_EDGE_WALL) sgnR = -1.0f;
        }
        const int py = ly + 1;
        const float hL = S.box[0][(py) * HX + l + 3], hR = S.box[0][(py) * HX + r + 3];
        const float qnL = sgnL * S.box[1][(py) * HX + l + 3], qtL = S.box[2][(py) * HX + l + 3];
        const float qnR = sgnR * S.box[1][(py) * HX + r + 3], qtR = S.box[2][(py) * HX + r + 3];
        const Face f = hll(g, dry, hL, qnL, qtL, sgnL * S.pu[py][l], S.pv[py][l], S.pc[py][l], hR, qnR, qtR,
                           sgnR * S.pu[py][r], S.pv[py][r], S.pc[py][r]);
        S.fx[0][ly][lf] = f.mass;
        S.fx[1][ly][lf] = f.normal;
        S.fx[2][ly][lf] = f.tangent;
    }
    // 3b. y-faces: face fy is the south face of cell fy (below = fy-1, above = fy)
    for (int i = tid; i < (TY + 1) * TX; i += SWE_THREADS) {
        const int lf = i / TX, lx = i % TX;
        const int gx = x0 + lx, gf = y0 + lf;
        if (gx >= nx || gf > ny) continue;
        int b = lf, t = lf + 1;       // primitive rows of the cells below and above
        float sgnB = 1.0f, sgnT = 1.0f;
        if (gf == 0) {
            b = t;
            if (a.edge[2] == VF_EDGE_WALL) sgnB = -1.0f;
        }
        if (gf == ny) {
            t = b;
            if (a.edge[3] == VF_EDGE_WALL) sgnT = -1.0f;
        }
        const int px = lx + 1;
        const float hB = S.box[0][(b) * HX + px + 3], hT = S.box[0][(t) * HX + px + 3];
        const float qnB = sgnB * S.box[2][(b) * HX + px + 3], qtB = S.box[1][(b) * HX + px + 3];
        const float qnT = sgnT * S.box[2][(t) * HX + px + 3], qtT = S.box[1][(t) * HX + px + 3];
        const Face f = hll(g, dry, hB, qnB, qtB, sgnB * S.pv[b][px], S.pu[b][px], S.pc[b][px], hT, qnT, qtT,
                           sgnT * S.pv[t][px], S.pu[t][px], S.pc[t][px]);
        S.fy[0][lf][lx] = f.mass;
        S.fy[1][lf][lx] = f.normal;
        S.fy[2][lf][lx] = f.tangent;
    }
    __syncthreads();

    // 4. the update (ShallowWater.java:206-235)
    int best = 0, clamps = 0;
    for (int i = tid; i < TY * TX; i += SWE_THREADS) {
        const int ly = i / TX, lx = i % TX;
        const int gx = x0 + lx, gy = y0 + ly;
        if (gx >= nx || gy >= ny) continue;
        const float h0 = S.box[0][(ly + 1) * HX + lx + 4], hu0 = S.box[1][(ly + 1) * HX + lx + 4], hv0 = S.box[2][(ly + 1) * HX + lx + 4];
        const float h = (h0 - rx * (S.fx[0][ly][lx + 1] - S.fx[0][ly][lx])) - ry * (S.fy[0][ly + 1][lx] - S.fy[0][ly][lx]);
        const float hu =
            (hu0 - rx * (S.fx[1][ly][lx + 1] - S.fx[1][ly][lx])) - ry * (S.fy[2][ly + 1][lx] - S.fy[2][ly][lx]);
        const float hv =
            (hv0 - rx * (S.fx[2][ly][lx + 1] - S.fx[2][ly][lx])) - ry * (S.fy[1][ly + 1][lx] - S.fy[1][ly][lx]);
        if (h < 0.0f) clamps++;
        const float nh = fmaxf(h, 0.0f);
        const int64_t c = (int64_t)gy * nx + gx;
        a.out[0][c] = nh;
        a.out[1][c] = hu;
        a.out[2][c] = hv;
        const float u = velocity(nh, hu, dry), w = velocity(nh, hv, dry);
        const float speed = fmaxf(fabsf(u), fabsf(w)) + sqrtf(g * nh);
        best = max(best, __float_as_int(speed));
        if (c == 0) {
            *a.speed_clear = 0;
            *a.budget_out = budget - ticks;
        }
    }
    // CTA reduction of the speed bits and the clamp count, then one atomic each
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
        clamps += __shfl_xor_sync(0xffffffffu, clamps, o);
    }
    if ((tid & 31) == 0) {
        S.red[tid >> 5] = best;
        if (clamps) atomicAdd(&S.clamps, clamps);
    }
    __syncthreads();
    if (tid == 0) {
        int m = 0;
        for (int w = 0; w < SWE_THREADS / 32; w++) m = max(m, S.red[w]);
        // only a filter: the buffer only grows within a step (ShallowWater.java:227-235)
        if (m > *(volatile int*)a.speed_out) atomicMax(a.speed_out, m);
        if (S.clamps) atomicAdd(a.clamped, S.clamps);
    }
    __syncthreads();   // the tile's shared memory is free for the next
    return true;
}

template <int TX_>
__device__ __forceinline__ SweShared<TX_>& swe_shared() {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const uint32_t mis = (uint32_t)__cvta_generic_to_shared(smem_raw) & 127u;
    return *reinterpret_cast<SweShared<TX_>*>(smem_raw + ((128u - mis) & 127u));
}

template <int TX_>
__device__ __forceinline__ void init_tile_barrier(SweShared<TX_>& S, bool tma) {
    if (threadIdx.x == 0 && tma) {
        const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&S.bar);
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
}

// One step, one CTA per tile (grid = tiles). Launched as a programmatic dependent of the previous step: its CTAs
// may become resident during that step's last wave, set up their barrier, and wait (griddepcontrol.wait: until
// the previous grid has completed and its stores are visible) before reading anything the previous step wrote.
template <int TX_>
__global__ void __launch_bounds__(SWE_THREADS) k_swe_tile(SweArgs a, const __grid_constant__ CUtensorMap tm_h,
                                                          const __grid_constant__ CUtensorMap tm_hu,
                                                          const __grid_constant__ CUtensorMap tm_hv) {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    SweShared<TX_>& S = swe_shared<TX_>();
    init_tile_barrier(S, a.use_tma);
    asm volatile("griddepcontrol.wait;" ::: "memory");
    swe_tile<TX_>(a, &tm_h, &tm_hu, &tm_hv, S, blockIdx.x, blockIdx.y, 0);
}

// ------------------------------------------------------------------ the fast mode's strip kernel
// One CTA of four warps per tile of 120 columns x 16 rows. The tile and a halo (columns x0-4 .. x0+123, rows
// y0-1 .. y0+16) land in shared memory by three 2D TMA loads; then every lane walks one column up the tile in
// registers: lane L of warp w holds column x0 + 30 w + L - 1, lanes 1..30 update their cell, lanes 0 and 31 only
// lend their state to their neighbours. A cell's west face is computed by its lane from its left neighbour's state
// (a shuffle), its east face is the right neighbour's west face (a shuffle), its south face was computed one row
// below and its north face is computed from the next row: every face once (twice where two warps meet, from the
// same inputs), the state read from shared memory once, and no shared-memory traffic for primitives or fluxes.
constexpr int STRIP_WARPS = 4;
constexpr int STRIP_COLS = 30 * STRIP_WARPS;   // columns a tile updates (a multiple of 4: the box's x stays aligned)
// 16 rows: 27.6 KB of tile a CTA, so eight CTAs fit an SM (at 4096^2 the fast step takes 0.124 ms against 0.129
// with 32 rows, whose 52 KB tiles left room for four)
constexpr int STRIP_ROWS = 16;
constexpr int STRIP_BW = 128;                  // box width: columns x0-4 .. x0+123
constexpr int STRIP_BH = STRIP_ROWS + 2;       // box height: rows y0-1 .. y0+ROWS

struct StripShared {
    float box[3][STRIP_BH * STRIP_BW];
    unsigned long long bar;
    int red[STRIP_WARPS];
    int clamps;
};

struct CellState {
    float h, qx, qy, u, v, c;   // depth, momenta, velocities, wave speed
};

__device__ __forceinline__ CellState cell_fast(float h, float qx, float qy, float g, float dry) {
    CellState q;
    q.h = h;
    q.qx = qx;
    q.qy = qy;
    const float inv = h > dry ? __fdividef(1.0f, h) : 0.0f;
    q.u = qx * inv;
    q.v = qy * inv;
    q.c = sqrt_fast(g * h);
    return q;
}

__device__ __forceinline__ CellState shfl_up_cell(const CellState& a) {
    const unsigned all = 0xffffffffu;
    CellState q;
    q.h = __shfl_up_sync(all, a.h, 1);
    q.qx = __shfl_up_sync(all, a.qx, 1);
    q.qy = __shfl_up_sync(all, a.qy, 1);
    q.u = __shfl_up_sync(all, a.u, 1);
    q.v = __shfl_up_sync(all, a.v, 1);
    q.c = __shfl_up_sync(all, a.c, 1);
    return q;
}

// The ghost of a cell across a side (ShallowWater.neighbour, ShallowWater.java:316-326): a wall negates the normal
// momentum (and so the normal velocity), an open side copies the cell.
__device__ __forceinline__ CellState ghost_x(CellState q, bool wall) {
    if (wall) {
        q.qx = -q.qx;
        q.u = -q.u;
    }
    return q;
}

__device__ __forceinline__ CellState ghost_y(CellState q, bool wall) {
    if (wall) {
        q.qy = -q.qy;
        q.v = -q.v;
    }
    return q;
}

// A cell's state and primitives in the exact arithmetic (velocity, sqrtf: IEEE division and square root).
__device__ __forceinline__ CellState cell_exact(float h, float qx, float qy, float g, float dry) {
    CellState q;
    q.h = h;
    q.qx = qx;
    q.qy = qy;
    q.u = velocity(h, qx, dry);
    q.v = velocity(h, qy, dry);
    q.c = sqrtf(g * h);
    return q;
}

// One CTA's column walk (k_swe_strip, step 2). INTERIOR: the tile and its halo lie inside the domain. EXACT: every
// operation as the tile kernel rounds it (the reference's strict f32); otherwise the fast mode's arithmetic.
template <bool INTERIOR, bool EXACT>
__device__ __forceinline__ void strip_walk(const SweArgs& a, StripShared& S, int x0, int y0, float g, float dry, float rx,
                                           float ry, int budget, int ticks, int& best, int& clamps) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nx = a.nx, ny = a.ny;
    const int cx = x0 + 30 * warp + lane - 1;        // this lane's column
    const int bc = 30 * warp + lane + 3;             // its column in the box
    const bool own = lane >= 1 && lane <= 30 && (INTERIOR || cx < nx);
    const bool wall_w = a.edge[0] == VF_EDGE_WALL, wall_e = a.edge[1] == VF_EDGE_WALL;
    const bool wall_s = a.edge[2] == VF_EDGE_WALL, wall_n = a.edge[3] == VF_EDGE_WALL;
    auto load = [&](int r) {
        const int i = r * STRIP_BW + bc;
        return EXACT ? cell_exact(S.box[0][i], S.box[1][i], S.box[2][i], g, dry)
                     : cell_fast(S.box[0][i], S.box[1][i], S.box[2][i], g, dry);
    };
    CellState prev = load(0);
    Face gs = {0.0f, 0.0f, 0.0f}, fw = {0.0f, 0.0f, 0.0f}, fe = {0.0f, 0.0f, 0.0f};
    for (int r = 1; r <= STRIP_ROWS + 1; r++) {
        const int y = y0 - 1 + r;   // this box row's row of the domain
        const CellState cur = load(r);
        // the face between rows y-1 and y (cur's south face, prev's north face), and this row's west face from the
        // left neighbour, together in paired fp32
        CellState bot = prev, top = cur;
        CellState left = shfl_up_cell(cur), right = cur;
        if (!INTERIOR) {
            if (y == 0) bot = ghost_y(cur, wall_s);
            if (y == ny) top = ghost_y(prev, wall_n);
            if (cx == 0) left = ghost_x(cur, wall_w);
            if (cx == nx) right = ghost_x(left, wall_e);
        }
        // the y-face (normal y) and the x-face (normal x); the fast mode pairs them, .x and .y
        Face gn, fwn;
        if (EXACT) {
            gn = hll(g, dry, bot.h, bot.qy, bot.qx, bot.v, bot.u, bot.c, top.h, top.qy, top.qx, top.v, top.u, top.c);
            fwn = hll(g, dry, left.h, left.qx, left.qy, left.u, left.v, left.c, right.h, right.qx, right.qy, right.u,
                      right.v, right.c);
        } else {
            const Face2 ff = hll_fast2(g, dry, f2(bot.h, left.h), f2(bot.qy, left.qx), f2(bot.qx, left.qy),
                                       f2(bot.v, left.u), f2(bot.u, left.v), f2(bot.c, left.c), f2(top.h, right.h),
                                       f2(top.qy, right.qx), f2(top.qx, right.qy), f2(top.v, right.u),
                                       f2(top.u, right.v), f2(top.c, right.c));
            gn = Face{ff.mass.x, ff.normal.x, ff.tangent.x};
            fwn = Face{ff.mass.y, ff.normal.y, ff.tangent.y};
        }
        if (r >= 2) {
            // the update of row y-1 (ShallowWater.java:206-235) from its four faces
            const int yu = y - 1;
            if (own && (INTERIOR || yu < ny)) {
                float h, hu, hv;
                if (EXACT) {
                    h = (prev.h - rx * (fe.mass - fw.mass)) - ry * (gn.mass - gs.mass);
                    hu = (prev.qx - rx * (fe.normal - fw.normal)) - ry * (gn.tangent - gs.tangent);
                    hv = (prev.qy - rx * (fe.tangent - fw.tangent)) - ry * (gn.normal - gs.normal);
                } else {
                    h = __fmaf_rn(-ry, gn.mass - gs.mass, __fmaf_rn(-rx, fe.mass - fw.mass, prev.h));
                    hu = __fmaf_rn(-ry, gn.tangent - gs.tangent, __fmaf_rn(-rx, fe.normal - fw.normal, prev.qx));
                    hv = __fmaf_rn(-ry, gn.normal - gs.normal, __fmaf_rn(-rx, fe.tangent - fw.tangent, prev.qy));
                }
                if (h < 0.0f) clamps++;
                const float nh = fmaxf(h, 0.0f);
                const int64_t c = (int64_t)yu * nx + cx;
                a.out[0][c] = nh;
                a.out[1][c] = hu;
                a.out[2][c] = hv;
                float speed;
                if (EXACT) {
                    const float u = velocity(nh, hu, dry), w = velocity(nh, hv, dry);
                    speed = fmaxf(fabsf(u), fabsf(w)) + sqrtf(g * nh);
                } else {
                    const float inv = nh > dry ? __fdividef(1.0f, nh) : 0.0f;
                    speed = fmaxf(fabsf(hu * inv), fabsf(hv * inv)) + sqrt_fast(g * nh);
                }
                best = max(best, __float_as_int(speed));
                if (!INTERIOR && c == 0) {
                    *a.speed_clear = 0;
                    *a.budget_out = budget - ticks;
                }
            }
        }
        gs = gn;
        // this row's x-faces for its update at the next row: its own west face, and the right neighbour's west face
        // as its east face
        fw = fwn;
        fe.mass = __shfl_down_sync(0xffffffffu, fw.mass, 1);
        fe.normal = __shfl_down_sync(0xffffffffu, fw.normal, 1);
        fe.tangent = __shfl_down_sync(0xffffffffu, fw.tangent, 1);
        prev = cur;
    }
}

template <bool EXACT>
__global__ void __launch_bounds__(STRIP_WARPS * 32) k_swe_strip(SweArgs a, const __grid_constant__ CUtensorMap tm_h,
                                                                    const __grid_constant__ CUtensorMap tm_hu,
                                                                    const __grid_constant__ CUtensorMap tm_hv) {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    extern __shared__ __align__(128) unsigned char strip_raw[];
    const uint32_t mis = (uint32_t)__cvta_generic_to_shared(strip_raw) & 127u;
    StripShared& S = *reinterpret_cast<StripShared*>(strip_raw + ((128u - mis) & 127u));
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0 && a.use_tma) {
        const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&S.bar);
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const int x0 = blockIdx.x * STRIP_COLS, y0 = blockIdx.y * STRIP_ROWS;
    const int nx = a.nx, ny = a.ny;
    // ShallowWater.java:184-192: the step from the fastest wave, in whole ticks, within the budget
    const float g = a.params[0], courant = a.params[1], dx = a.params[2], dy = a.params[3], dry = a.params[4];
    const float fastest = __int_as_float(__ldcg(a.speed_in));
    const float allowed = fminf((courant * fminf(dx, dy)) / fmaxf(fastest, 1e-30f), 2000.0f);
    int ticks = (int)(allowed * 1000000.0f);
    const int budget = __ldcg(a.budget_in);
    if (budget < ticks) ticks = budget;
    const float dt = (float)ticks * (float)(1.0 / 1000000.0);
    const float rx = dt / dx;
    const float ry = dt / dy;
    // 1. stage the tile and its halo
    bool loaded = true;
    if (tid == 0) S.clamps = 0;
    if (a.use_tma) {
        if (tid == 0) {
            const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&S.bar);
            const uint32_t bytes = 3u * STRIP_BH * STRIP_BW * 4u;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
            const CUtensorMap* maps[3] = {&tm_h, &tm_hu, &tm_hv};
            const int bx = x0 - 4, by = y0 - 1;   // bx is a multiple of 4: 16-byte aligned
            for (int f = 0; f < 3; f++) {
                const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&S.box[f][0]);
                asm volatile(
                    "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
                    "[%4];" ::"r"(dst),
                    "l"(maps[f]), "r"(bx), "r"(by), "r"(bar)
                    : "memory");
            }
        }
        loaded = wait_barrier(&S.bar, 0, a.status);
    } else {
        for (int i = tid; i < STRIP_BH * STRIP_BW; i += STRIP_WARPS * 32) {
            const int ly = i / STRIP_BW, lx = i % STRIP_BW;
            const int gx = x0 - 4 + lx, gy = y0 - 1 + ly;
            const bool in = gx >= 0 && gx < nx && gy >= 0 && gy < ny;
            const int64_t c = (int64_t)gy * nx + gx;
            for (int f = 0; f < 3; f++) S.box[f][i] = in ? __ldcg(a.in[f] + c) : 0.0f;
        }
    }
    if (!__syncthreads_and(loaded)) return;   // a TMA that never landed: the status says so, nothing is written

    // 2. the column walk: tiles that touch no side of the domain skip every ghost and bounds test
    int best = 0, clamps = 0;
    const bool interior = x0 >= 1 && x0 + STRIP_COLS + 1 <= nx && y0 >= 1 && y0 + STRIP_ROWS + 1 <= ny;
    if (interior)
        strip_walk<true, EXACT>(a, S, x0, y0, g, dry, rx, ry, budget, ticks, best, clamps);
    else
        strip_walk<false, EXACT>(a, S, x0, y0, g, dry, rx, ry, budget, ticks, best, clamps);
    // 3. the CTA's fastest wave and clamp count, one atomic each
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
        clamps += __shfl_xor_sync(0xffffffffu, clamps, o);
    }
    if (lane == 0) {
        S.red[warp] = best;
        if (clamps) atomicAdd(&S.clamps, clamps);
    }
    __syncthreads();
    if (tid == 0) {
        int m = 0;
        for (int w = 0; w < STRIP_WARPS; w++) m = max(m, S.red[w]);
        if (m > *(volatile int*)a.speed_out) atomicMax(a.speed_out, m);
        if (S.clamps) atomicAdd(a.clamped, S.clamps);
    }
}

// ------------------------------------------------------------------ diagnostics (Diagnostics.of)

struct DiagPart {
    double volume, min_depth, max_depth, max_speed, max_froude, max_wave;
    int non_finite, negative, wet;
};

// The next step's wave speed from a state the host or another kernel changed: bits of the largest
// max(|u|, |v|) + sqrt(g h), the same per-cell expression the step's update computes (ShallowWater.java:236-241).
__global__ void __launch_bounds__(256) k_swe_speed(const float* h, const float* hu, const float* hv, int64_t n,
                                                   const float* params, int* speed) {
    const float g = params[0], dry = params[4];
    int best = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float d = h[i];
        const float u = velocity(d, hu[i], dry), w = velocity(d, hv[i], dry);
        best = max(best, __float_as_int(fmaxf(fabsf(u), fabsf(w)) + sqrtf(g * d)));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0 && best > 0) atomicMax(speed, best);
}

// Coarse cell (i, j) of the box [x0, x0 + cnx) x [y0, y0 + cny) = the mean of fine cells (2i..2i+1, 2j..2j+1)
// counted from the fine patch's cell (fx0, fy0).
// One device word from a kernel argument: the budget written in stream order, without a host wait.
__global__ void k_swe_set_word(int* p, int v) { *p = v; }

__global__ void k_swe_restrict(const float* const* fine, int fnx, int fx0, int fy0, float* const* coarse, int ccnx,
                               int x0, int y0, int cnx, int cny) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (int64_t)cnx * cny) return;
    const int i = (int)(k % cnx), j = (int)(k / cnx);
    const int64_t f = (int64_t)(fy0 + 2 * j) * fnx + fx0 + 2 * i;
    const int64_t c = (int64_t)(y0 + j) * ccnx + x0 + i;
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const float* a = fine[q];
        coarse[q][c] = 0.25f * ((a[f] + a[f + 1]) + (a[f + fnx] + a[f + fnx + 1]));
    }
}

// Fine patch cell (fi, fj) = coarse cell (x0 + fi/2, y0 + fj/2), the coarse index clamped into its grid.
__global__ void k_swe_prolong(const float* const* coarse, int ccnx, int ccny, int x0, int y0, float* const* fine, int fnx,
                              int fny) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (int64_t)fnx * fny) return;
    const int fi = (int)(k % fnx), fj = (int)(k / fnx);
    const int ci = min(max(x0 + fi / 2, 0), ccnx - 1), cj = min(max(y0 + fj / 2, 0), ccny - 1);
    const int64_t c = (int64_t)cj * ccnx + ci;
#pragma unroll
    for (int q = 0; q < 3; q++) fine[q][k] = coarse[q][c];
}

// Per tile of t x t cells: the largest relative depth jump to the east or north neighbour,
// (|h(i+1,j) - h(i,j)| + |h(i,j+1) - h(i,j)|) / max(h(i,j), dry), as float bits (atomicMax).
__global__ void k_swe_jump(const float* h, int nx, int ny, int t, int tiles_x, float dry, int* out) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (int64_t)nx * ny) return;
    const int i = (int)(k % nx), j = (int)(k / nx);
    const float d = h[k];
    const float ex = i < nx - 1 ? fabsf(h[k + 1] - d) : 0.0f;
    const float ny_ = j < ny - 1 ? fabsf(h[k + nx] - d) : 0.0f;
    const float jump = (ex + ny_) / fmaxf(d, dry);
    atomicMax(&out[(j / t) * tiles_x + i / t], __float_as_int(jump));
}

__global__ void __launch_bounds__(256) k_swe_diag(const float* h, const float* hu, const float* hv, int64_t n,
                                                  double g, double dry, DiagPart* parts) {
    DiagPart p{0.0, INFINITY, 0.0, 0.0, 0.0, 0.0, 0, 0, 0};
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const float hk = h[k], uk = hu[k], vk = hv[k];
        if (!isfinite(hk) || !isfinite(uk) || !isfinite(vk)) {
            p.non_finite++;
            continue;
        }
        if (hk < 0) p.negative++;
        p.volume += hk;
        p.max_depth = fmax(p.max_depth, (double)hk);
        if ((double)hk <= dry) continue;
        p.wet++;
        p.min_depth = fmin(p.min_depth, (double)hk);
        const double u = (double)uk / hk, v = (double)vk / hk;
        const double c = sqrt(g * hk);
        const double speed = sqrt(u * u + v * v);
        p.max_speed = fmax(p.max_speed, speed);
        if (hk >= 1e-3) p.max_froude = fmax(p.max_froude, speed / c);
        p.max_wave = fmax(p.max_wave, fmax(fabs(u), fabs(v)) + c);
    }
    __shared__ DiagPart sp[256];
    sp[threadIdx.x] = p;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            DiagPart& a = sp[threadIdx.x];
            const DiagPart& b = sp[threadIdx.x + s];
            a.volume += b.volume;
            a.min_depth = fmin(a.min_depth, b.min_depth);
            a.max_depth = fmax(a.max_depth, b.max_depth);
            a.max_speed = fmax(a.max_speed, b.max_speed);
            a.max_froude = fmax(a.max_froude, b.max_froude);
            a.max_wave = fmax(a.max_wave, b.max_wave);
            a.non_finite += b.non_finite;
            a.negative += b.negative;
            a.wet += b.wet;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) parts[blockIdx.x] = sp[0];
}


// A 2D tensor map over one nx x ny f32 field with an hx x hy box; false if TMA cannot take it
// (row pitch not a multiple of 16 bytes, or an unaligned base).
bool make_map(CUtensorMap* m, const float* base, int nx, int ny, int hx, int hy) {
    EncodeTiled enc = tensor_map_encoder();
    if (!enc) return false;
    if (((uintptr_t)base & 15) || ((int64_t)nx * 4) % 16 != 0) return false;
    cuuint64_t dims[2] = {(cuuint64_t)nx, (cuuint64_t)ny};
    cuuint64_t strides[1] = {(cuuint64_t)nx * 4};
    cuuint32_t box[2] = {(cuuint32_t)hx, (cuuint32_t)hy};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void*)base, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

}  // namespace

// ------------------------------------------------------------------ the handle

struct vf_swe {
    int nx, ny;
    int edges[4];
    int64_t cells;
    cudaStream_t stream = nullptr;
    DeviceBuffer state[2];    // 3 fields each
    DeviceBuffer small;       // speed[3], budget[2], clamped, params[5] (as ints/floats)
    DeviceBuffer status, diag;
    int32_t* host_words = nullptr;   // pinned: the budget and the status word read back together
    CUtensorMap maps[2][2][3];   // [tile width 64, 32][state][field]
    CUtensorMap smaps[2][3];     // the fast mode's strip boxes: [state][field]
    bool tma = false;
    int tile_w = 64;             // 64 or 32: the staged tile kernel; 0: the column walk over strips (k_swe_strip)
    bool pdl = true;             // steps launched as programmatic dependents of the previous step
    bool exact = true;           // false: the fast mode's arithmetic (vf_swe_set_exact)
    // PatchSimulation.java:52-56
    int64_t clock_now = 0;
    int32_t clock_outstanding = 0;
    int64_t dispatched = 0;
    int64_t total_steps = 0;
    int64_t last_step = 0;
    float host_params[5];
    Profiler prof;
};

namespace {

int* small_i(vf_swe* h) { return h->small.as<int>(); }
int* speed_slot(vf_swe* h, int k) { return small_i(h) + k; }          // 0..2
int* budget_slot(vf_swe* h, int k) { return small_i(h) + 3 + k; }     // 3..4
int* clamped_ptr(vf_swe* h) { return small_i(h) + 5; }                // 5
float* params_ptr(vf_swe* h) { return h->small.as<float>() + 8; }     // 8..12

float* field(vf_swe* h, int s, int f) { return h->state[s].as<float>() + (int64_t)f * h->cells; }

int32_t swe_params_check(const int32_t* params, int32_t n, float out[5]) {
    VF_REQUIRE(params && n == 5, VF_EINVAL, "ShallowWater.params has 5 words, got %d", n);
    for (int k = 0; k < 5; k++) out[k] = bits_to_float(params[k]);
    // ShallowWater.paramsAllowingInstability refuses a Courant number that is not positive (262-264);
    // above 1/2 is the caller's choice (params vs paramsAllowingInstability).
    VF_REQUIRE(out[1] > 0, VF_EINVAL, "a Courant number must be positive, got %g", out[1]);
    return VF_OK;
}

// One dispatch: step k of the rotation (PatchSimulation.dispatch, PatchSimulation.java:197-205).
int32_t dispatch(vf_swe* h) {
    const int64_t k = h->dispatched;
    const int si = (int)(k % 2), so = (int)((k + 1) % 2);
    SweArgs a;
    for (int f = 0; f < 3; f++) {
        a.in[f] = field(h, si, f);
        a.out[f] = field(h, so, f);
    }
    a.params = params_ptr(h);
    a.speed_in = speed_slot(h, (int)(k % 3));
    a.speed_out = speed_slot(h, (int)((k + 1) % 3));
    a.speed_clear = speed_slot(h, (int)((k + 2) % 3));
    a.budget_in = budget_slot(h, si);
    a.budget_out = budget_slot(h, so);
    a.clamped = clamped_ptr(h);
    a.status = h->status.as<uint32_t>();
    a.nx = h->nx;
    a.ny = h->ny;
    for (int e = 0; e < 4; e++) a.edge[e] = h->edges[e];
    a.use_tma = h->tma ? 1 : 0;
    const int wide = h->tile_w == 64;
    const bool tile = h->exact && h->tile_w != 0;
    CUtensorMap* m = tile ? h->maps[wide ? 0 : 1][si] : h->smaps[si];
    void* args[] = {&a, &m[0], &m[1], &m[2]};
    cudaLaunchConfig_t cfg = {};
    if (tile) {
        cfg.gridDim = dim3(div_up(h->nx, h->tile_w), div_up(h->ny, SWE_TY));
        cfg.blockDim = dim3(SWE_THREADS);
        cfg.dynamicSmemBytes = wide ? sizeof(SweShared<64>) + 128 : sizeof(SweShared<32>) + 128;
    } else {
        cfg.gridDim = dim3(div_up(h->nx, STRIP_COLS), div_up(h->ny, STRIP_ROWS));
        cfg.blockDim = dim3(STRIP_WARPS * 32);
        cfg.dynamicSmemBytes = sizeof(StripShared) + 128;
    }
    cfg.stream = h->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = h->pdl ? 1 : 0;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const void* fn = tile ? (wide ? (const void*)k_swe_tile<64> : (const void*)k_swe_tile<32>)
                          : h->exact ? (const void*)k_swe_strip<true> : (const void*)k_swe_strip<false>;
    h->prof.begin(tile ? "k_swe_tile" : h->exact ? "k_swe_strip" : "k_swe_strip_fast", h->stream);
    const cudaError_t e = cudaLaunchKernelExC(&cfg, fn, args);
    h->prof.end(h->stream);
    VF_TRY_CUDA(e);
    h->dispatched++;
    return VF_OK;
}

// The budget left in slot and the device status word, in one host wait.
int32_t read_budget(vf_swe* h, int slot, int32_t* out, uint32_t* status) {
    VF_TRY_CUDA(cudaMemcpyAsync(h->host_words, budget_slot(h, slot), 4, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaMemcpyAsync(h->host_words + 1, h->status.ptr, 4, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    *out = h->host_words[0];
    if (status) *status = (uint32_t)h->host_words[1];
    return VF_OK;
}

// Stream-ordered: the steps dispatched after it read the new budget; no host wait.
int32_t write_budget(vf_swe* h, int slot, int32_t v) {
    VF_LAUNCH(h->prof, "k_swe_set_word", h->stream, k_swe_set_word, 1, 1, 0, budget_slot(h, slot), v);
    return VF_OK;
}

// A nonzero device status (read back with the budget): cleared, and reported as the error it is.
int32_t status_error(vf_swe* h, uint32_t st) {
    if (!st) return VF_OK;
    VF_TRY_CUDA(cudaMemsetAsync(h->status.ptr, 0, 4, h->stream));
    set_error("a kernel flagged device status 0x%x", st);
    return (st & ST_TIMEOUT) ? VF_ETIMEOUT : VF_EDEVICE;
}

int32_t status_swe(vf_swe* h) {
    uint32_t st = 0;
    VF_TRY_CUDA(cudaMemcpyAsync(&st, h->status.ptr, 4, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return status_error(h, st);
}

// ShallowWater.fastestWave (ShallowWater.java:287-295), on the host.
int32_t fastest_wave_bits(const float* h, const float* hu, const float* hv, int64_t n, double g, double dry) {
    float fastest = 0.0f;
    for (int64_t k = 0; k < n; k++) {
        float u = (double)h[k] > dry ? hu[k] / h[k] : 0.0f;
        float w = (double)h[k] > dry ? hv[k] / h[k] : 0.0f;
        float c = (float)std::sqrt(g * (double)h[k]);
        float s = std::fmax(std::fabs(u), std::fabs(w)) + c;
        if (std::isnan(s) || std::isnan(fastest)) fastest = NAN;
        else fastest = fastest > s ? fastest : s;
    }
    int32_t b;
    memcpy(&b, &fastest, 4);
    return b;
}

}  // namespace

extern "C" {

int32_t vf_swe_create(int32_t nx, int32_t ny, const int32_t edges[4], vf_swe** out) {
    VF_REQUIRE(out && edges, VF_EINVAL, "null argument");
    *out = nullptr;
    VF_REQUIRE(nx >= 1 && ny >= 1, VF_EINVAL, "a patch needs at least one cell each way, got %d x %d", nx, ny);
    for (int e = 0; e < 4; e++)
        VF_REQUIRE(edges[e] == VF_EDGE_WALL || edges[e] == VF_EDGE_OPEN, VF_EINVAL, "every side of a patch needs an edge");
    int32_t rc = require_device();
    if (rc) return rc;
    vf_swe* h = new vf_swe();
    h->nx = nx;
    h->ny = ny;
    for (int e = 0; e < 4; e++) h->edges[e] = edges[e];
    h->cells = (int64_t)nx * ny;
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        set_error("cudaStreamCreate failed");
        return VF_ECUDA;
    }
    if ((rc = h->state[0].alloc((size_t)3 * h->cells * 4)) || (rc = h->state[1].alloc((size_t)3 * h->cells * 4)) ||
        (rc = h->small.alloc(64)) || (rc = h->status.alloc(16)) || (rc = h->diag.alloc(sizeof(DiagPart) * 1184))) {
        vf_swe_destroy(h);
        return rc;
    }
    if (cudaMallocHost(&h->host_words, 16) != cudaSuccess) {
        h->host_words = nullptr;
        vf_swe_destroy(h);
        set_error("cudaMallocHost(16) failed");
        return VF_ENOMEM;
    }
    for (DeviceBuffer* b : {&h->state[0], &h->state[1], &h->small, &h->status}) cudaMemsetAsync(b->ptr, 0, b->bytes, h->stream);
    if (cudaFuncSetAttribute(k_swe_tile<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(SweShared<64>) + 128) != cudaSuccess ||
        cudaFuncSetAttribute(k_swe_tile<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(SweShared<32>) + 128) != cudaSuccess ||
        cudaFuncSetAttribute(k_swe_strip<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(StripShared) + 128) != cudaSuccess ||
        cudaFuncSetAttribute(k_swe_strip<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(StripShared) + 128) != cudaSuccess) {
        vf_swe_destroy(h);
        set_error("cannot give the shallow-water kernel %zu bytes of shared memory", sizeof(SweShared<64>));
        return VF_ECUDA;
    }
    bool tma = true;
    for (int s = 0; s < 2; s++)
        for (int f = 0; f < 3; f++)
            tma = tma && make_map(&h->maps[0][s][f], field(h, s, f), nx, ny, Tile<64>::HX, Tile<64>::HY) &&
                  make_map(&h->maps[1][s][f], field(h, s, f), nx, ny, Tile<32>::HX, Tile<32>::HY) &&
                  make_map(&h->smaps[s][f], field(h, s, f), nx, ny, STRIP_BW, STRIP_BH);
    h->tma = tma;
    if (!tma) {
        memset(h->maps, 0, sizeof h->maps);
        memset(h->smaps, 0, sizeof h->smaps);
    }
    h->tile_w = 64;
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
        vf_swe_destroy(h);
        set_error("clearing buffers failed");
        return VF_ECUDA;
    }
    *out = h;
    return VF_OK;
}

int32_t vf_swe_load(vf_swe* h, const float* hcell, const float* hu, const float* hv, const int32_t* params,
                    int32_t nparams) {
    VF_REQUIRE(h && hcell && hu && hv, VF_EINVAL, "null argument");
    float p[5];
    int32_t rc = swe_params_check(params, nparams, p);
    if (rc) return rc;
    memcpy(h->host_params, p, sizeof p);
    h->dispatched = 0;
    h->total_steps = 0;
    h->last_step = 0;
    h->clock_now = 0;
    h->clock_outstanding = 0;
    const float* src[3] = {hcell, hu, hv};
    for (int f = 0; f < 3; f++)
        VF_TRY_CUDA(cudaMemcpyAsync(field(h, 0, f), src[f], (size_t)h->cells * 4, cudaMemcpyHostToDevice, h->stream));
    int32_t small[16] = {0};
    small[0] = fastest_wave_bits(hcell, hu, hv, h->cells, (double)p[0], (double)p[4]);   // PatchSimulation.java:100-102
    memcpy(small + 8, p, sizeof p);
    VF_TRY_CUDA(cudaMemcpyAsync(h->small.ptr, small, sizeof small, cudaMemcpyHostToDevice, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return VF_OK;
}

int32_t vf_swe_params(vf_swe* h, const int32_t* params, int32_t nparams) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    float p[5];
    int32_t rc = swe_params_check(params, nparams, p);
    if (rc) return rc;
    memcpy(h->host_params, p, sizeof p);
    VF_TRY_CUDA(cudaMemcpyAsync(params_ptr(h), p, sizeof p, cudaMemcpyHostToDevice, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return VF_OK;
}

// PatchSimulation.advance (PatchSimulation.java:120-145). The clock is the host's i64 tick count:
// grant gives up to 2^31-1 ticks to the device as its budget; settle moves the clock by what was spent.
int32_t vf_swe_advance(vf_swe* h, int64_t ticks, int32_t max_steps, int32_t* steps_out, int64_t* spent,
                       int64_t* behind) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    VF_REQUIRE(ticks >= 0 && max_steps >= 0, VF_EINVAL, "ticks and maxSteps must be >= 0");
    const int64_t before = h->clock_now;
    const int64_t want = (before + ticks) - h->clock_now;
    const int32_t granted = (int32_t)(want < 0 ? 0 : want > 2147483647LL ? 2147483647LL : want);
    h->clock_outstanding = granted;
    int32_t rc = write_budget(h, (int)(h->dispatched % 2), granted);
    if (rc) return rc;
    int32_t left = granted;
    int32_t steps = 0;
    bool read = false;
    uint32_t st = 0;
    while (left > 0 && steps < max_steps) {
        const int32_t batch =
            h->last_step > 0 ? (int32_t)std::min<int64_t>(max_steps - steps, ((int64_t)left + h->last_step - 1) / h->last_step)
                             : 1;
        for (int s = 0; s < batch; s++)
            if ((rc = dispatch(h))) return rc;
        steps += batch;
        int32_t now = 0;
        if ((rc = read_budget(h, (int)(h->dispatched % 2), &now, &st))) return rc;
        read = true;
        if (now > 0 && now < left) h->last_step = (left - now) / batch;
        left = now;
    }
    h->clock_now += h->clock_outstanding - left;   // settle
    h->clock_outstanding = 0;
    h->total_steps += steps;
    if (steps_out) *steps_out = steps;
    if (spent) *spent = h->clock_now - before;
    if (behind) *behind = left;
    return read ? status_error(h, st) : status_swe(h);
}

int32_t vf_swe_read(vf_swe* h, float* hcell, float* hu, float* hv) {
    VF_REQUIRE(h && hcell && hu && hv, VF_EINVAL, "null argument");
    const int s = (int)(h->dispatched % 2);
    float* dst[3] = {hcell, hu, hv};
    for (int f = 0; f < 3; f++)
        VF_TRY_CUDA(cudaMemcpyAsync(dst[f], field(h, s, f), (size_t)h->cells * 4, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return status_swe(h);
}

int32_t vf_swe_fastest_wave(vf_swe* h, double* out) {
    VF_REQUIRE(h && out, VF_EINVAL, "null argument");
    int32_t b = 0;
    VF_TRY_CUDA(cudaMemcpyAsync(&b, speed_slot(h, (int)(h->dispatched % 3)), 4, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    *out = (double)bits_to_float(b);
    return VF_OK;
}

int32_t vf_swe_clamped(vf_swe* h, int32_t* out) {
    VF_REQUIRE(h && out, VF_EINVAL, "null argument");
    VF_TRY_CUDA(cudaMemcpyAsync(out, clamped_ptr(h), 4, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return VF_OK;
}

int64_t vf_swe_now(const vf_swe* h) { return h ? h->clock_now : 0; }

int64_t vf_swe_steps(const vf_swe* h) { return h ? h->total_steps : 0; }

int32_t vf_swe_dispatch(vf_swe* h, int32_t n) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    VF_REQUIRE(n >= 0, VF_EINVAL, "n must be >= 0");
    for (int k = 0; k < n; k++) {
        int32_t rc = dispatch(h);
        if (rc) return rc;
    }
    return VF_OK;
}

int64_t vf_swe_dispatched(const vf_swe* h) { return h ? h->dispatched : 0; }

// The snapshot's body: the 16-word device block (speed words in their rotation, budget words, clamp count, params),
// the host clock, dispatch count, step total and last step's ticks, then h, hu, hv of the current state.
int32_t vf_swe_snapshot(vf_swe* h, void* buf, int64_t cap, int64_t* size) {
    VF_REQUIRE(h && size, VF_EINVAL, "null argument");
    const size_t fields = (size_t)3 * h->cells * 4;
    const uint64_t payload = 64 + 4 * 8 + fields;
    *size = (int64_t)(sizeof(SnapHeader) + payload);
    if (!buf) return VF_OK;
    VF_REQUIRE(cap >= *size, VF_EINVAL, "a snapshot of this patch takes %lld bytes, the buffer has %lld",
               (long long)*size, (long long)cap);
    VF_REQUIRE(h->clock_outstanding == 0, VF_ESTATE, "a grant is outstanding");
    char* body = static_cast<char*>(buf) + sizeof(SnapHeader);
    VF_TRY_CUDA(cudaMemcpyAsync(body, h->small.ptr, 64, cudaMemcpyDeviceToHost, h->stream));
    const int64_t clock[4] = {h->clock_now, h->dispatched, h->total_steps, h->last_step};
    memcpy(body + 64, clock, sizeof clock);
    const int s = (int)(h->dispatched % 2);
    for (int f = 0; f < 3; f++)
        VF_TRY_CUDA(cudaMemcpyAsync(body + 96 + (size_t)f * h->cells * 4, field(h, s, f), (size_t)h->cells * 4,
                                    cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    int32_t rc = status_swe(h);
    if (rc) return rc;
    const int32_t edges = h->edges[0] | h->edges[1] << 8 | h->edges[2] << 16 | h->edges[3] << 24;
    SnapHeader hd = snap_header(SNAP_SWE, h->nx, h->ny, 1, edges, h->cells, h->total_steps, payload);
    hd.checksum = fnv1a(body, payload);
    memcpy(buf, &hd, sizeof hd);
    return VF_OK;
}

int32_t vf_swe_restore(vf_swe* h, const void* buf, int64_t size) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    const int32_t edges = h->edges[0] | h->edges[1] << 8 | h->edges[2] << 16 | h->edges[3] << 24;
    SnapHeader want = snap_header(SNAP_SWE, h->nx, h->ny, 1, edges, h->cells, 0, 64 + 4 * 8 + (size_t)3 * h->cells * 4);
    SnapHeader got;
    int32_t rc = snap_check(buf, size, want, &got);
    if (rc) return rc;
    const char* body = static_cast<const char*>(buf) + sizeof(SnapHeader);
    int32_t small[16];
    memcpy(small, body, sizeof small);
    float p[5];
    if ((rc = swe_params_check(small + 8, 5, p))) return rc;
    int64_t clock[4];
    memcpy(clock, body + 64, sizeof clock);
    VF_REQUIRE(clock[1] >= 0 && clock[2] >= 0 && clock[3] >= 0, VF_EINVAL, "a snapshot with negative counts");
    const int s = (int)(clock[1] % 2);
    for (int f = 0; f < 3; f++)
        VF_TRY_CUDA(cudaMemcpyAsync(field(h, s, f), body + 96 + (size_t)f * h->cells * 4, (size_t)h->cells * 4,
                                    cudaMemcpyHostToDevice, h->stream));
    VF_TRY_CUDA(cudaMemcpyAsync(h->small.ptr, small, sizeof small, cudaMemcpyHostToDevice, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    memcpy(h->host_params, p, sizeof p);
    h->clock_now = clock[0];
    h->dispatched = clock[1];
    h->total_steps = clock[2];
    h->last_step = clock[3];
    h->clock_outstanding = 0;
    return VF_OK;
}

int32_t vf_swe_set_tile_width(vf_swe* h, int32_t width) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    VF_REQUIRE(width == 0 || width == 32 || width == 64, VF_EINVAL, "a tile is 32 or 64 cells wide (0: strips), got %d",
               width);
    h->tile_w = width;
    return VF_OK;
}

int32_t vf_swe_tile_width(const vf_swe* h) { return h ? h->tile_w : 0; }

int32_t vf_swe_set_exact(vf_swe* h, int32_t on) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    h->exact = on != 0;
    return VF_OK;
}

int32_t vf_swe_exact(const vf_swe* h) { return h && h->exact ? 1 : 0; }

int32_t vf_swe_set_overlap(vf_swe* h, int32_t on) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    h->pdl = on != 0;
    return VF_OK;
}

int32_t vf_swe_write_budget(vf_swe* h, int32_t slot, int32_t ticks) {
    VF_REQUIRE(h && (slot == 0 || slot == 1), VF_EINVAL, "budget slot is 0 or 1");
    return write_budget(h, slot, ticks);
}

int32_t vf_swe_read_budget(vf_swe* h, int32_t slot, int32_t* ticks) {
    VF_REQUIRE(h && ticks && (slot == 0 || slot == 1), VF_EINVAL, "budget slot is 0 or 1");
    uint32_t st = 0;
    int32_t rc = read_budget(h, slot, ticks, &st);
    return rc ? rc : status_error(h, st);
}

int32_t vf_swe_diagnostics(vf_swe* h, double g, double dry, double dt, double dx, double dy, double out[9]) {
    VF_REQUIRE(h && out, VF_EINVAL, "null argument");
    const int s = (int)(h->dispatched % 2);
    const int blocks = 1184;
    k_swe_diag<<<blocks, 256, 0, h->stream>>>(field(h, s, 0), field(h, s, 1), field(h, s, 2), h->cells,
                                              g, dry,
                                              h->diag.as<DiagPart>());
    VF_CHECK_LAUNCH();
    std::vector<DiagPart> parts(blocks);
    VF_TRY_CUDA(cudaMemcpyAsync(parts.data(), h->diag.ptr, sizeof(DiagPart) * blocks, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    DiagPart t{0.0, INFINITY, 0.0, 0.0, 0.0, 0.0, 0, 0, 0};
    for (const DiagPart& p : parts) {
        t.volume += p.volume;
        t.min_depth = std::fmin(t.min_depth, p.min_depth);
        t.max_depth = std::fmax(t.max_depth, p.max_depth);
        t.max_speed = std::fmax(t.max_speed, p.max_speed);
        t.max_froude = std::fmax(t.max_froude, p.max_froude);
        t.max_wave = std::fmax(t.max_wave, p.max_wave);
        t.non_finite += p.non_finite;
        t.negative += p.negative;
        t.wet += p.wet;
    }
    out[0] = t.volume * dx * dy;
    out[1] = t.wet == 0 ? 0 : t.min_depth;
    out[2] = t.max_depth;
    out[3] = t.max_speed;
    out[4] = t.max_froude;
    out[5] = t.max_wave * dt / std::fmin(dx, dy);
    out[6] = t.non_finite;
    out[7] = t.negative;
    out[8] = t.wet;
    return VF_OK;
}

void* vf_swe_stream(vf_swe* h) { return h ? (void*)h->stream : nullptr; }

int32_t vf_swe_profile(vf_swe* h, int32_t enable) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    h->prof.reset();
    h->prof.on = enable != 0;
    return VF_OK;
}

int32_t vf_swe_profile_read(vf_swe* h, int32_t index, char* name, size_t cap, double* total_ms, int64_t* launches) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    return h->prof.read(index, name, cap, total_ms, launches);
}

int64_t vf_swe_launches(const vf_swe* h) { return h ? h->prof.launches : 0; }

int32_t vf_swe_on_gpu(const vf_swe* h) { return h ? 1 : 0; }

void vf_swe_destroy(vf_swe* h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (DeviceBuffer* b : {&h->state[0], &h->state[1], &h->small, &h->status, &h->diag}) b->release();
    if (h->host_words) cudaFreeHost(h->host_words);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}


// ------------------------------------------------------------------ the state on the device

int32_t vf_swe_state(vf_swe* h, float** hcell, float** hu, float** hv) {
    VF_REQUIRE(h && hcell && hu && hv, VF_EINVAL, "null argument");
    const int s = (int)(h->dispatched % 2);
    *hcell = field(h, s, 0);
    *hu = field(h, s, 1);
    *hv = field(h, s, 2);
    return VF_OK;
}

int32_t vf_swe_measure_speed(vf_swe* h) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    const int s = (int)(h->dispatched % 2);
    int* slot = speed_slot(h, (int)(h->dispatched % 3));
    VF_TRY_CUDA(cudaMemsetAsync(slot, 0, 4, h->stream));
    VF_LAUNCH(h->prof, "k_swe_speed", h->stream, k_swe_speed, std::max(1, std::min(div_up(h->cells, 256), sm_count() * 8)), 256,
              0, field(h, s, 0), field(h, s, 1), field(h, s, 2), h->cells, params_ptr(h), slot);
    return VF_OK;   // the next dispatch, on the same stream, reads the word
}

namespace {

// The three current fields of a handle as a device array of pointers (a small upload on the handle's stream).
struct FieldPtrs {
    DeviceBuffer buf;
    int32_t make(vf_swe* h) {
        const int s = (int)(h->dispatched % 2);
        float* p[3] = {field(h, s, 0), field(h, s, 1), field(h, s, 2)};
        int32_t rc = buf.alloc(sizeof p);
        if (rc) return rc;
        VF_TRY_CUDA(cudaMemcpyAsync(buf.ptr, p, sizeof p, cudaMemcpyHostToDevice, h->stream));
        return VF_OK;
    }
};

}  // namespace

int32_t vf_swe_restrict(vf_swe* fine, vf_swe* coarse) {
    VF_REQUIRE(fine && coarse, VF_EINVAL, "null handle");
    VF_REQUIRE(fine->nx == 2 * coarse->nx && fine->ny == 2 * coarse->ny, VF_EINVAL,
               "a %d x %d grid restricts to %d x %d, not %d x %d", fine->nx, fine->ny, fine->nx / 2, fine->ny / 2,
               coarse->nx, coarse->ny);
    VF_TRY_CUDA(cudaStreamSynchronize(fine->stream));
    FieldPtrs f, c;
    int32_t rc;
    if ((rc = f.make(fine)) || (rc = c.make(coarse))) return rc;
    VF_TRY_CUDA(cudaStreamSynchronize(fine->stream));
    VF_LAUNCH(coarse->prof, "k_swe_restrict", coarse->stream, k_swe_restrict, div_up(coarse->cells, 256), 256, 0,
              f.buf.as<const float*>(), fine->nx, 0, 0, c.buf.as<float*>(), coarse->nx, 0, 0, coarse->nx, coarse->ny);
    VF_TRY_CUDA(cudaStreamSynchronize(coarse->stream));
    return vf_swe_measure_speed(coarse);
}

int32_t vf_swe_prolong(vf_swe* coarse, int32_t x0, int32_t y0, vf_swe* fine) {
    VF_REQUIRE(fine && coarse, VF_EINVAL, "null handle");
    VF_REQUIRE(fine->nx % 2 == 0 && fine->ny % 2 == 0, VF_EINVAL, "a patch of even size, got %d x %d", fine->nx, fine->ny);
    VF_TRY_CUDA(cudaStreamSynchronize(coarse->stream));
    FieldPtrs f, c;
    int32_t rc;
    if ((rc = f.make(fine)) || (rc = c.make(coarse))) return rc;
    VF_TRY_CUDA(cudaStreamSynchronize(coarse->stream));
    VF_LAUNCH(fine->prof, "k_swe_prolong", fine->stream, k_swe_prolong, div_up(fine->cells, 256), 256, 0,
              c.buf.as<const float*>(), coarse->nx, coarse->ny, x0, y0, f.buf.as<float*>(), fine->nx, fine->ny);
    VF_TRY_CUDA(cudaStreamSynchronize(fine->stream));
    return vf_swe_measure_speed(fine);
}

int32_t vf_swe_restrict_patch(vf_swe* fine, int32_t fx0, int32_t fy0, vf_swe* coarse, int32_t x0, int32_t y0,
                              int32_t nx, int32_t ny) {
    VF_REQUIRE(fine && coarse, VF_EINVAL, "null handle");
    VF_REQUIRE(nx >= 1 && ny >= 1 && fx0 >= 0 && fy0 >= 0 && fx0 + 2 * nx <= fine->nx && fy0 + 2 * ny <= fine->ny,
               VF_EINVAL, "%d x %d coarse cells from fine cell (%d, %d) leave the %d x %d patch", nx, ny, fx0, fy0,
               fine->nx, fine->ny);
    VF_REQUIRE(x0 >= 0 && y0 >= 0 && x0 + nx <= coarse->nx && y0 + ny <= coarse->ny, VF_EINVAL,
               "coarse cells [%d, %d) x [%d, %d) leave the %d x %d grid", x0, x0 + nx, y0, y0 + ny, coarse->nx, coarse->ny);
    VF_TRY_CUDA(cudaStreamSynchronize(fine->stream));
    FieldPtrs f, c;
    int32_t rc;
    if ((rc = f.make(fine)) || (rc = c.make(coarse))) return rc;
    VF_TRY_CUDA(cudaStreamSynchronize(fine->stream));
    VF_LAUNCH(coarse->prof, "k_swe_restrict", coarse->stream, k_swe_restrict, div_up((int64_t)nx * ny, 256), 256, 0,
              f.buf.as<const float*>(), fine->nx, fx0, fy0, c.buf.as<float*>(), coarse->nx, x0, y0, nx, ny);
    VF_TRY_CUDA(cudaStreamSynchronize(coarse->stream));
    return VF_OK;
}

int32_t vf_swe_copy_state(vf_swe* dst, vf_swe* src) {
    VF_REQUIRE(dst && src, VF_EINVAL, "null handle");
    VF_REQUIRE(dst->nx == src->nx && dst->ny == src->ny, VF_EINVAL, "grids differ: %d x %d and %d x %d", dst->nx,
               dst->ny, src->nx, src->ny);
    VF_TRY_CUDA(cudaStreamSynchronize(src->stream));
    const int sd = (int)(dst->dispatched % 2), ss = (int)(src->dispatched % 2);
    for (int f = 0; f < 3; f++)
        VF_TRY_CUDA(cudaMemcpyAsync(field(dst, sd, f), field(src, ss, f), (size_t)src->cells * 4, cudaMemcpyDeviceToDevice,
                                    dst->stream));
    return vf_swe_measure_speed(dst);
}

int32_t vf_swe_jump_indicator(vf_swe* h, int32_t tile, float* out, int32_t ntiles) {
    VF_REQUIRE(h && out && tile >= 1, VF_EINVAL, "null argument or tile < 1");
    const int tx = (h->nx + tile - 1) / tile, ty = (h->ny + tile - 1) / tile;
    VF_REQUIRE(ntiles == tx * ty, VF_EINVAL, "%d tiles of %d cells cover the grid, got %d", tx * ty, tile, ntiles);
    DeviceBuffer d;
    int32_t rc = d.alloc((size_t)ntiles * 4);
    if (rc) return rc;
    VF_TRY_CUDA(cudaMemsetAsync(d.ptr, 0, (size_t)ntiles * 4, h->stream));
    const int s = (int)(h->dispatched % 2);
    VF_LAUNCH(h->prof, "k_swe_jump", h->stream, k_swe_jump, div_up(h->cells, 256), 256, 0, field(h, s, 0), h->nx, h->ny,
              tile, tx, h->host_params[4], d.as<int>());
    VF_TRY_CUDA(cudaMemcpyAsync(out, d.ptr, (size_t)ntiles * 4, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return VF_OK;
}

}  // extern "C"
