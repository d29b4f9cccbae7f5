// mpm3.cu -- the vf_mpm3_* C-ABI: ParticleSimulation3 (vexelray-sim-fluid-gui/.../gui/
// ParticleSimulation3.java) over Flip3Step's pass list (Flip3Step.java:81-118), on one CUDA stream.
//
// One step, with the default flags (sort every step, tiled scatter):
//   [sort]    brick scan -> cell scan -> permute -> stable fix-up       (counts from the last G2P)
//   clear     the node windows the scatter two steps ago touched in this grid buffer
//   scatter   k_p2g3_tile  (or k_p2g3_atomic / k_p2g3_warp after a dense clear)
//   grid      fused into k_g2p3_tile (or k_grid3_dense for the other schedules); with VF_TENSION the colour, its
//             blurs, the stress and k_grid3_tension write the velocity grid, which every G2P then reads
//   advect    k_g2p3_tile  gathers each particle through the sort's permutation, writes it to its
//             sorted slot in the other particle set, and counts its new key for the next sort
#include <algorithm>
#include <cmath>
#include <mutex>
#include <vector>

#include "mpm3_kernels.cuh"
#include "profiler.cuh"
#include "snapshot.cuh"

using namespace vf;

// A snapshot's param block (seven Flip3.params words and a zero pad) and the flags it must agree on: the physics
// flags, not the scatter schedule or the sort switch, so a run can resume under another schedule.
constexpr int SNAP3_WORDS = 8;
constexpr uint32_t SNAP3_FLAGS = ~(uint32_t)(VF_P2G_MASK | VF_NO_SORT);

struct vf_mpm3 {
    int nx, ny, nz, np;
    uint32_t flags;
    int p2g;
    bool sort;
    Dims3 d;
    int nbricks;
    int64_t nkeys, nodes, stride;
    cudaStream_t stream = nullptr;
    DeviceBuffer part[2];
    int cur = 0;
    DeviceBuffer key, perm;
    DeviceBuffer cell_count, cell_start, cursor;
    DeviceBuffer brick_count, brick_start;
    DeviceBuffer active[2];   // the non-empty bricks of the step that scattered into grid[g]
    DeviceBuffer n_active;    // int[4]: the non-empty bricks of each list, then each list's gather item counter
    DeviceBuffer grid[2];
    DeviceBuffer vel;
    DeviceBuffer params;
    DeviceBuffer status;
    DeviceBuffer scratch;     // readouts
    DeviceBuffer pdiag;       // the particle diagnostics' histograms, made on first use
    DeviceBuffer nominal;     // the smallest positive mass loaded, as float bits (ParticleSimulation3.java:248-253)
    DeviceBuffer fixed;       // the exact schedule's grid: int64 [4][nodes], FIXED3_BITS fractional bits
    bool tension = false;     // VF_TENSION: Tension3's passes between the scatter and the grid
    DeviceBuffer colour[2];   // the blurs' ping-pong colour planes, nodes floats each
    DeviceBuffer stress;      // txx tyy tzz txy txz tyz, nodes floats each
    // sparse node storage (vf_mpm3_prepare_sparse): grid[g] is a pool of pool_cap bricks of 8^3 nodes and page[g]
    // maps the domain's brick positions (pnx x pny x pnz) into it, rebuilt by every scatter into grid[g]
    bool sparse = false;
    int pool_cap = 0;
    int pnx = 0, pny = 0, pnz = 0;
    int npages = 0;
    DeviceBuffer page[2], mark;
    DeviceBuffer n_used;      // int[2]: the slots the last scatter into each pool took
    DeviceBuffer view;        // sparse: the last grid unpacked into the dense box for readouts, made on first use
    bool view_fresh = false;  // `view` holds the last grid
    bool fixed_valid = false; // `fixed` holds the last scatter's sums
    Params3 hparams{};
    int64_t steps = 0;
    int64_t passes_run = 0;   // steps run through vf_mpm3_run / advance, for grid parity
    int grid_last = 1;        // the grid buffer the last scatter wrote
    // what each grid buffer needs before the next scatter into it: 0 clean, 1 sparse (clear the
    // windows of active[g]), 2 dense (memset)
    int grid_dirty[2] = {0, 0};
    bool counted = false;     // cell/brick counts and key/rank hold the current positions' keys
    // The fused step (k_g2p2g3): the gather of step k and the scatter of step k+1 in one kernel. `fused` selects it
    // (vf_mpm3_set_fused, where it applies: the sorted tiled schedule, dense storage, no tension); `ahead` says the
    // grid buffer grid_last holds the scatter of the CURRENT particles (the next step's), so readouts of the last
    // step's grid look in the other buffer. Off by default: at the 3D configuration it measured no faster than the
    // separate tiled passes.
    bool fused = false;
    bool fuse_wanted = false;
    bool ahead = false;
    bool sorted_valid = false;
    bool loaded = false;
    Profiler prof;
    // vf_mpm3_set_graph: two steps captured as one CUDA graph from a host state that recurs every two steps, and
    // replayed while the state before a pair is the one it was captured from
    bool use_graph = false;
    cudaGraphExec_t pair = nullptr;
    uint64_t pair_sig = 0;
    int64_t pair_launches = 0;
};

struct vf_mpm3_prepared {
    vf_mpm3* sim = nullptr;
    bool taken = false;
};

namespace {

int32_t upload_params(vf_mpm3* h, const int32_t* params, int32_t nparams) {
    VF_REQUIRE(params && nparams >= 6, VF_EINVAL, "Flip3.params has at least 6 words, got %d", nparams);
    float w[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int k = 0; k < 7 && k < nparams; k++) w[k] = bits_to_float(params[k]);
    // Flip3.params refuses these (Flip3.java:98-101)
    VF_REQUIRE(w[0] > 0 && w[4] >= 0 && w[5] > 0, VF_EINVAL,
               "dt > 0, bulk >= 0 and rho0 > 0, got dt %g, bulk %g, rho0 %g", w[0], w[4], w[5]);
    Params3 p;
    p.dt = w[0];
    p.gx = w[1];
    p.gy = w[2];
    p.gz = w[3];
    p.bulk = w[4];
    p.rho0 = w[5];
    p.sigma = w[6];
    p.tait = (h->flags & VF_EOS_TAIT) ? 1 : 0;
    p.sticky = (int)((h->flags & VF_WALL_STICKY_MASK) >> VF_WALL_STICKY_SHIFT);
    h->hparams = p;
    VF_TRY_CUDA(cudaMemcpyAsync(h->params.ptr, &p, sizeof p, cudaMemcpyHostToDevice, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return VF_OK;
}

Step3 make_step(vf_mpm3* h) {
    Step3 s{};
    s.out = h->part[h->cur].as<float>();
    s.in = s.out;
    s.stride = h->stride;
    s.np = h->np;
    s.perm = nullptr;
    s.vel = h->vel.as<float4>();
    s.params = h->params.as<Params3>();
    s.d = h->d;
    s.status = h->status.as<uint32_t>();
    s.key = h->key.as<int>();
    s.cell_count = h->cell_count.as<int>();
    s.brick_count = h->brick_count.as<int>();
    s.cell_start = h->cell_start.as<int>();
    s.brick_start = h->brick_start.as<int>();
    s.nkeys = h->nkeys;
    s.nbricks = h->nbricks;
    // the tiled G2P's items per brick: bricks hold about 2,048 particles or more, and the G2P keeps four CTAs an SM
    // busy; the 256^3 configuration's 2,000 bricks need no split, a 17k-particle drop's dozen take eight items each
    s.g2p_split = (int)std::min<int64_t>(8, std::max<int64_t>(1, (int64_t)sm_count() * 4 / std::max(1, h->np / 2048)));
    s.sparse = h->sparse ? 1 : 0;
    s.pool_cap = h->pool_cap;
    s.pnx = h->pnx;
    s.pny = h->pny;
    s.pnz = h->pnz;
    return s;
}

int persistent_blocks(int per_sm) { return sm_count() * per_sm; }

bool fuse_applies(const vf_mpm3* h) { return h->p2g == VF_P2G_TILE && h->sort && !h->tension && !h->sparse; }

// The grid buffer holding the last step's scatter (what grid(), the snapshot and the device pointers show).
int ref_grid(const vf_mpm3* h) { return h->ahead ? h->grid_last ^ 1 : h->grid_last; }

// Forgets a scatter made ahead for the current particles (before anything changes them, the params, the schedule,
// or runs passes on its own): the buffer it went into is cleared densely before its next use.
void drop_ahead(vf_mpm3* h) {
    if (!h->ahead) return;
    h->grid_dirty[h->grid_last] = 2;
    h->grid_last ^= 1;
    h->passes_run--;
    h->ahead = false;
}

// VF_P2G_AUTO: the schedule measured fastest for the handle's size. Below about 600k particles the tiled scatter,
// one warp per unit of 8x8x1 cells, leaves much of the GPU idle: the
// warp-aggregated scatter over the dense grid is 1.8x faster at 17k particles in a 40^3 box and 1.2x at 358k in
// 96^3. Above that, or on grids where the dense passes (clear, grid update: 48 B a node) would cost more than the
// particles, the tile wins (1.05x at 0.9M in 128^3, 1.35x at 7.2M in 256^3). Sparse storage always runs the tile.
constexpr int64_t AUTO_TILE_PARTICLES = 600000;
constexpr int64_t AUTO_TILE_NODES = int64_t(1) << 22;
int resolve_p2g(int schedule, int64_t particles, int64_t nodes, bool sparse) {
    if (schedule != VF_P2G_AUTO) return schedule;
    return sparse || particles >= AUTO_TILE_PARTICLES || nodes >= AUTO_TILE_NODES ? VF_P2G_TILE : VF_P2G_WARP;
}

// The grid update into `vel` for the step that scattered into grid[g]: Flip3.grid, or with tension the colour,
// its blurs, the stress and Flip3.gridWithTension (Flip3Step.java:88-109).
int32_t grid_pass(vf_mpm3* h, Step3& s, int g) {
    s.grid = h->grid[g].as<float4>();
    if (!h->tension) {
        VF_LAUNCH(h->prof, "k_grid3_dense", h->stream, k_grid3_dense, div_up(h->nodes, 256), 256, 0, s);
        return VF_OK;
    }
    const int blocks = div_up(h->nodes, 256);
    float* c[2] = {h->colour[0].as<float>(), h->colour[1].as<float>()};
    for (int k = 0; k < TENSION3_BLURS; k++) {
        h->prof.begin(k == 0 ? "k_tension3_colour" : "k_tension3_blur", h->stream);
        const cudaError_t e = launch_tension3_blur(k == 0, k == 0 ? (const void*)s.grid : (const void*)c[(k - 1) % 2],
                                                   c[k % 2], s.params, s.d, h->stream);
        h->prof.end(h->stream);
        VF_TRY_CUDA(e);
    }
    const float* colour = c[(TENSION3_BLURS - 1) % 2];
    h->prof.begin("k_tension3_stress", h->stream);
    const cudaError_t e = launch_tension3_stress(colour, h->stress.as<float>(), s.d, h->stream);
    h->prof.end(h->stream);
    VF_TRY_CUDA(e);
    VF_LAUNCH(h->prof, "k_grid3_tension", h->stream, k_grid3_tension, blocks, 256, 0, s, colour, h->stress.as<float>());
    return VF_OK;
}

// The nominal mass of the current set's masses, on the device: the smallest positive one, FLT_MAX if none.
int32_t measure_nominal(vf_mpm3* h) {
    VF_TRY_CUDA(fill_f32(h->nominal.as<float>(), 1, 3.402823466e+38f, h->stream));
    k_min_positive3<<<std::max(1, std::min(div_up(h->np, 256), sm_count() * 4)), 256, 0, h->stream>>>(
        h->part[h->cur].as<float>() + (int64_t)M * h->stride, h->np, h->nominal.as<unsigned>());
    VF_CHECK_LAUNCH();
    return VF_OK;
}

// Zero the counts so the next count pass starts clean (after positions changed under the
// counts of a G2P that counted ahead).
int32_t reset_counts(vf_mpm3* h) {
    VF_TRY_CUDA(cudaMemsetAsync(h->cell_count.ptr, 0, h->cell_count.bytes, h->stream));
    VF_TRY_CUDA(cudaMemsetAsync(h->brick_count.ptr, 0, h->brick_count.bytes, h->stream));
    h->counted = false;
    return VF_OK;
}

// The sort passes, leaving perm = sorted slot -> particle of the current set. `g` is the grid
// buffer this step scatters into; its brick list is rebuilt here (after its old windows are cleared).
int32_t run_sort(vf_mpm3* h, int g, bool will_scatter, bool fused_fixup) {
    Step3 s = make_step(h);
    if (!h->counted) {
        VF_LAUNCH(h->prof, "k_key_count3", h->stream, k_key_count3, div_up(h->np, 256), 256, 0, s);
    }
    // the old windows of grid[g] must be cleared before its brick list is overwritten; a sort with
    // no scatter after it leaves the grid alone and marks it for a dense clear instead
    if (h->grid_dirty[g] == 1 && !will_scatter) h->grid_dirty[g] = 2;
    s.grid = h->grid[g].as<float4>();
    s.active = h->active[g].as<int>();
    s.n_active = h->n_active.as<int>() + g;
    if (h->grid_dirty[g] == 1) {
        if (h->sparse)
            VF_LAUNCH(h->prof, "k_pool_clear3", h->stream, k_pool_clear3, persistent_blocks(8), 256, 0, s.grid,
                      h->n_used.as<int>() + g);
        else
            VF_LAUNCH(h->prof, "k_clear_bricks3", h->stream, k_clear_bricks3, persistent_blocks(8), 256, 0, s);
        h->grid_dirty[g] = 0;
    }
    int* active = h->active[g].as<int>();
    int* n_active = h->n_active.as<int>() + g;
    VF_LAUNCH(h->prof, "k_brick_scan", h->stream, k_brick_scan, 1, 1024, 0, h->brick_count.as<int>(), h->brick_start.as<int>(), active, n_active,
                                           h->nbricks);
    if (h->sparse && will_scatter) {
        // the page of grid[g] for this step: the node bricks the non-empty cell bricks' windows reach
        VF_LAUNCH(h->prof, "k_pool_mark3", h->stream, k_pool_mark3, persistent_blocks(2), 256, 0, s, h->mark.as<int>());
        VF_LAUNCH(h->prof, "k_pool_page3", h->stream, k_pool_page3, 1, 1024, 0, h->mark.as<int>(), h->page[g].as<int>(),
                  h->npages, h->n_used.as<int>() + g, h->pool_cap, h->status.as<uint32_t>());
    }
    VF_LAUNCH(h->prof, "k_cell_scan", h->stream, k_cell_scan, persistent_blocks(4), 512, 0, h->cell_count.as<int>(),
              h->cell_start.as<int>(), h->cursor.as<int>(),
                                                          h->brick_start.as<int>(), active, n_active);
    VF_LAUNCH(h->prof, "k_permute_cursor", h->stream, k_permute_cursor, div_up(h->np, 256 * PERMUTE_PER), 256, 0, h->key.as<int>(),
              h->cursor.as<int>(), h->perm.as<int>(), h->np, h->nkeys, h->status.as<uint32_t>());
    // the tiled scatter puts each cell's run in order itself; everything else needs the fix-up pass
    if (!fused_fixup)
        VF_LAUNCH(h->prof, "k_fixup_bricks", h->stream, k_fixup_bricks, persistent_blocks(2), 512, 12288 * sizeof(int),
                  h->perm.as<int>(), h->cell_start.as<int>(), h->brick_start.as<int>(), active, n_active);
    h->counted = false;
    h->sorted_valid = true;
    return VF_OK;
}

// One step's passes. mask selects them (VF3_PASS_*). The grid buffer alternates per step.
int32_t run_passes(vf_mpm3* h, uint32_t mask, bool count_next) {
    const int g = (int)(h->passes_run & 1);
    const bool sort = (mask & VF3_PASS_SORT) && h->sort;
    const bool tile = h->p2g == VF_P2G_TILE && sort;
    if ((mask & VF3_PASS_ADVECT) && h->counted && !sort) {
        // counts made ahead for positions this advect is about to move, and no sort to consume them
        int32_t rc = reset_counts(h);
        if (rc) return rc;
    }
    if (sort) {
        int32_t rc = run_sort(h, g, (mask & VF3_PASS_SCATTER) != 0, tile && (mask & VF3_PASS_SCATTER));
        if (rc) return rc;
    }
    Step3 s = make_step(h);
    s.grid = h->grid[g].as<float4>();
    s.active = h->active[g].as<int>();
    s.n_active = h->n_active.as<int>() + g;
    s.page = h->sparse ? h->page[g].as<int>() : nullptr;
    if (sort) {
        s.perm = h->perm.as<int>();
        s.out = h->part[h->cur ^ 1].as<float>();
    }
    if (mask & VF3_PASS_CLEAR) {
        if (tile) {
            if (h->grid_dirty[g] == 2) VF_TRY_CUDA(cudaMemsetAsync(s.grid, 0, h->grid[g].bytes, h->stream));
            // a sparse-dirty buffer was cleared by run_sort before its list was replaced
        } else {
            VF_TRY_CUDA(cudaMemsetAsync(s.grid, 0, h->grid[g].bytes, h->stream));
        }
        h->grid_dirty[g] = 0;
    }
    if (mask & VF3_PASS_SCATTER) {
        if (tile) {
            h->prof.begin("k_p2g3_tile", h->stream);
            const cudaError_t e = launch_p2g3_tile(persistent_blocks(2), s, h->stream);
            h->prof.end(h->stream);
            VF_TRY_CUDA(e);
        } else if (h->p2g == VF_P2G_WARP) {
            VF_LAUNCH(h->prof, "k_p2g3_warp", h->stream, k_p2g3_warp, div_up(h->np, 256), 256, 0, s);
        } else if (h->p2g == VF_P2G_FIXED) {
            if (!h->fixed.ptr) {
                int32_t rc = h->fixed.alloc((size_t)4 * h->nodes * sizeof(long long));
                if (rc) return rc;
            }
            VF_TRY_CUDA(cudaMemsetAsync(h->fixed.ptr, 0, h->fixed.bytes, h->stream));
            VF_LAUNCH(h->prof, "k_p2g3_fixed", h->stream, k_p2g3_fixed, div_up(h->np, 256), 256, 0, s,
                      h->fixed.as<unsigned long long>());
            VF_LAUNCH(h->prof, "k_fixed_to_grid3", h->stream, k_fixed_to_grid3, div_up(h->nodes, 256), 256, 0,
                      h->fixed.as<long long>(), s.grid, h->nodes);
        } else {
            VF_LAUNCH(h->prof, "k_p2g3_atomic", h->stream, k_p2g3_atomic, div_up(h->np, 256), 256, 0, s);
        }
        VF_CHECK_LAUNCH();
        h->grid_dirty[g] = tile ? 1 : 2;
        h->grid_last = g;
        h->view_fresh = false;
        h->fixed_valid = h->p2g == VF_P2G_FIXED;
    }
    if (mask & VF3_PASS_ADVECT) {
        s.count_next = count_next ? 1 : 0;
        int32_t rc;
        if (tile) {
            // the tiled G2P updates the grid itself, unless tension's force needs the whole grid first
            if (h->tension) {
                if ((rc = grid_pass(h, s, g))) return rc;
                s.vel_ready = 1;
            }
            s.work = h->n_active.as<int>() + 2 + g;
            VF_LAUNCH(h->prof, "k_g2p3_tile", h->stream, k_g2p3_tile, persistent_blocks(4), 256, 0, s);
        } else {
            if ((rc = grid_pass(h, s, g))) return rc;
            VF_LAUNCH(h->prof, "k_g2p3", h->stream, k_g2p3, div_up(h->np, 256), 256, 0, s);
        }
        if (sort) h->cur ^= 1;
        h->counted = count_next;
    } else if (mask & VF3_PASS_GRID) {
        int32_t rc = grid_pass(h, s, g);
        if (rc) return rc;
    }
    if (sort && !(mask & VF3_PASS_ADVECT)) {
        // the particles were not moved to their sorted slots; apply the permutation as a copy
        VF_LAUNCH(h->prof, "k_gather_fields", h->stream, k_gather_fields, div_up(h->np, 256), 256, 0, s.in, s.out,
                  s.perm, h->np, h->stride, (int)NF3);
        h->cur ^= 1;
    }
    if (mask & VF3_PASS_SCATTER) h->passes_run++;
    return VF_OK;
}

// The host state a step's launches and their arguments depend on (everything else is in device memory or fixed
// at creation): which particle set is current, whether the counts were made ahead, the grid parity and each grid
// buffer's clear, the schedule, and whether the exact schedule's buffer exists.
uint64_t step_sig(const vf_mpm3* h) {
    return (uint64_t)h->cur | (uint64_t)h->counted << 1 | (uint64_t)(h->passes_run & 1) << 2 |
           (uint64_t)h->grid_dirty[0] << 3 | (uint64_t)h->grid_dirty[1] << 5 | (uint64_t)h->grid_last << 7 |
           (uint64_t)h->p2g << 8 | (uint64_t)(h->fixed.ptr != nullptr) << 12 | (uint64_t)h->fused << 13 |
           (uint64_t)h->ahead << 14 | 1ull << 63;
}

constexpr uint32_t STEP_PASSES = VF3_PASS_SORT | VF3_PASS_CLEAR | VF3_PASS_SCATTER | VF3_PASS_GRID | VF3_PASS_ADVECT;

// The fused step's first scatter: the current particles sorted and scattered by the tiled schedule (which also
// puts each cell's run in order), into the buffer the next scatter takes. Afterwards grid_last holds the scatter
// of the current particles and the permutation is theirs.
int32_t fused_prologue(vf_mpm3* h) {
    const int g = (int)(h->passes_run & 1);
    int32_t rc = run_sort(h, g, true, true);
    if (rc) return rc;
    Step3 s = make_step(h);
    s.grid = h->grid[g].as<float4>();
    s.active = h->active[g].as<int>();
    s.n_active = h->n_active.as<int>() + g;
    s.perm = h->perm.as<int>();
    if (h->grid_dirty[g] == 2) VF_TRY_CUDA(cudaMemsetAsync(s.grid, 0, h->grid[g].bytes, h->stream));
    h->grid_dirty[g] = 0;
    h->prof.begin("k_p2g3_tile", h->stream);
    const cudaError_t e = launch_p2g3_tile(persistent_blocks(2), s, h->stream);
    h->prof.end(h->stream);
    VF_TRY_CUDA(e);
    h->grid_dirty[g] = 1;   // its footprint: the windows of active[g]
    h->grid_last = g;
    h->view_fresh = false;
    h->fixed_valid = false;
    h->passes_run++;
    h->ahead = true;
    return VF_OK;
}

// The sort of the current particles by the keys the last fused kernel counted, in fused mode: the brick list it
// makes (active[grid_last]) is both the next fused kernel's work and the footprint of the scatter already in
// grid[grid_last]. No stable fix-up: the fused kernel's sums are atomic, so the order within a cell does not matter.
int32_t fused_sort(vf_mpm3* h) {
    const int g = h->grid_last;
    int* active = h->active[g].as<int>();
    int* n_active = h->n_active.as<int>() + g;
    VF_LAUNCH(h->prof, "k_brick_scan", h->stream, k_brick_scan, 1, 1024, 0, h->brick_count.as<int>(),
              h->brick_start.as<int>(), active, n_active, h->nbricks);
    VF_LAUNCH(h->prof, "k_cell_scan", h->stream, k_cell_scan, persistent_blocks(4), 512, 0, h->cell_count.as<int>(),
              h->cell_start.as<int>(), h->cursor.as<int>(), h->brick_start.as<int>(), active, n_active);
    VF_LAUNCH(h->prof, "k_permute_cursor", h->stream, k_permute_cursor, div_up(h->np, 256 * PERMUTE_PER), 256, 0, h->key.as<int>(),
              h->cursor.as<int>(), h->perm.as<int>(), h->np, h->nkeys, h->status.as<uint32_t>());
    h->counted = false;
    h->sorted_valid = true;
    return VF_OK;
}

// One fused step: [the prologue scatter, or the sort] then k_g2p2g3, which gathers from grid[grid_last], writes the
// advected particles to their sorted slots in the other set, scatters them into the other grid buffer (cleared
// here over its last footprint) and counts their keys.
int32_t fused_step(vf_mpm3* h) {
    int32_t rc = h->ahead ? fused_sort(h) : fused_prologue(h);
    if (rc) return rc;
    const int gi = h->grid_last, go = gi ^ 1;
    Step3 s = make_step(h);
    if (h->grid_dirty[go] == 1) {
        s.grid = h->grid[go].as<float4>();
        s.active = h->active[go].as<int>();
        s.n_active = h->n_active.as<int>() + go;
        VF_LAUNCH(h->prof, "k_clear_bricks3", h->stream, k_clear_bricks3, persistent_blocks(8), 256, 0, s);
    } else if (h->grid_dirty[go] == 2) {
        VF_TRY_CUDA(cudaMemsetAsync(h->grid[go].ptr, 0, h->grid[go].bytes, h->stream));
    }
    h->grid_dirty[go] = 0;
    s.grid = h->grid[gi].as<float4>();
    s.active = h->active[gi].as<int>();
    s.n_active = h->n_active.as<int>() + gi;
    s.perm = h->perm.as<int>();
    s.out = h->part[h->cur ^ 1].as<float>();
    s.count_next = 1;
    h->prof.begin("k_g2p2g3", h->stream);
    const cudaError_t e = launch_g2p2g3(persistent_blocks(fused_blocks_per_sm()), s, h->grid[go].as<float4>(), h->stream);
    h->prof.end(h->stream);
    VF_TRY_CUDA(e);
    h->cur ^= 1;
    h->grid_last = go;
    h->grid_dirty[go] = 1;   // its footprint list is made by the next fused sort, into active[go]
    h->passes_run++;
    h->counted = true;
    h->view_fresh = false;
    h->fixed_valid = false;
    return VF_OK;
}

// One step of advance(): fused where it applies, else Flip3Step's passes.
int32_t step_once(vf_mpm3* h) {
    if (h->fused) return fused_step(h);
    drop_ahead(h);
    return run_passes(h, STEP_PASSES, h->sort);
}

// Two steps into h->pair by stream capture, then launched once. The host state the capture advanced is put back
// if the capture fails, and the steps are left to run uncaptured.
int32_t capture_pair(vf_mpm3* h, uint64_t sig) {
    const int cur = h->cur, dirty0 = h->grid_dirty[0], dirty1 = h->grid_dirty[1], last = h->grid_last;
    const bool counted = h->counted, sorted = h->sorted_valid, fresh = h->view_fresh, fixed = h->fixed_valid;
    const int64_t passes = h->passes_run, launches = h->prof.launches;
    if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return VF_ECUDA;
    }
    const bool ahead = h->ahead;
    int32_t rc = step_once(h);
    if (!rc) rc = step_once(h);
    cudaGraph_t graph = nullptr;
    const cudaError_t end = cudaStreamEndCapture(h->stream, &graph);
    cudaGraphExec_t exec = nullptr;
    if (!rc && end == cudaSuccess && step_sig(h) == sig &&
        cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
        cudaGraphDestroy(graph);
        if (h->pair) cudaGraphExecDestroy(h->pair);
        h->pair = exec;
        h->pair_sig = sig;
        h->pair_launches = h->prof.launches - launches;
        VF_TRY_CUDA(cudaGraphLaunch(h->pair, h->stream));
        return VF_OK;
    }
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    h->cur = cur;
    h->grid_dirty[0] = dirty0;
    h->grid_dirty[1] = dirty1;
    h->grid_last = last;
    h->ahead = ahead;
    h->counted = counted;
    h->sorted_valid = sorted;
    h->view_fresh = fresh;
    h->fixed_valid = fixed;
    h->passes_run = passes;
    h->prof.launches = launches;
    return VF_ECUDA;
}

int32_t check_status(vf_mpm3* h) {
    uint32_t st = 0;
    VF_TRY_CUDA(cudaMemcpyAsync(&st, h->status.ptr, 4, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    if (st) {
        VF_TRY_CUDA(cudaMemsetAsync(h->status.ptr, 0, 4, h->stream));
        set_error("a kernel flagged device status 0x%x (1 index out of range, 2 wait timeout, 4 sort rank, 8 the "
                  "sparse grid's brick pool is full)", st);
        return VF_EDEVICE;
    }
    return VF_OK;
}

// The last scatter's grid as the dense box: grid[grid_last], or for sparse storage the pool unpacked through its
// page into `view` (allocated on first use, unpacked once per scatter).
int32_t last_grid(vf_mpm3* h, float4** out) {
    if (!h->sparse) {
        *out = h->grid[ref_grid(h)].as<float4>();
        return VF_OK;
    }
    if (!h->view.ptr) {
        int32_t rc = h->view.alloc((size_t)h->nodes * 16);
        if (rc) return rc;
        VF_TRY_CUDA(cudaMemsetAsync(h->view.ptr, 0, h->view.bytes, h->stream));
    }
    if (!h->view_fresh) {
        Step3 s = make_step(h);
        s.grid = h->grid[h->grid_last].as<float4>();
        s.page = h->page[h->grid_last].as<int>();
        k_pool_unpack3<<<div_up(h->nodes, 256), 256, 0, h->stream>>>(s, h->view.as<float4>());
        VF_CHECK_LAUNCH();
        h->view_fresh = true;
    }
    *out = h->view.as<float4>();
    return VF_OK;
}

int32_t field_pointer(vf_mpm3* h, int32_t field, float** ptr, int64_t* n) {
    if (field >= VF3_X && field <= VF3_C22) {
        *ptr = h->part[h->cur].as<float>() + (int64_t)field * h->stride;
        *n = h->np;
        return VF_OK;
    }
    set_error("no particle field %d", field);
    return VF_EINVAL;
}

}  // namespace

extern "C" {

}  // extern "C"

namespace {

int32_t prepare3(int32_t nx, int32_t ny, int32_t nz, int32_t particles, uint32_t flags, int32_t pool_bricks,
                 vf_mpm3_prepared** out) {
    VF_REQUIRE(out, VF_EINVAL, "out is null");
    *out = nullptr;
    VF_REQUIRE(particles >= 1, VF_EINVAL, "a step needs particles, got %d", particles);
    VF_REQUIRE(nx >= 3 && ny >= 3 && nz >= 3, VF_EINVAL, "a 3D grid needs at least three nodes each way, got %d x %d x %d",
               nx, ny, nz);
    {
        // brick-major cell keys (bricks of 8^3 stencil cells) and node indices are int32 in the kernels
        const int64_t bricks = (int64_t)((nx - 2 + 7) / 8) * ((ny - 2 + 7) / 8) * ((nz - 2 + 7) / 8);
        VF_REQUIRE(bricks * 512 <= INT32_MAX && (int64_t)nx * ny <= INT32_MAX, VF_EINVAL,
                   "a %d x %d x %d grid is too large: its cell keys (%lld) would not fit an int32", nx, ny, nz,
                   (long long)(bricks * 512));
    }
    int p2g = (int)((flags & VF_P2G_MASK) >> VF_P2G_SHIFT);
    VF_REQUIRE(p2g <= VF_P2G_AUTO, VF_EINVAL, "no scatter schedule %d", p2g);
    p2g = resolve_p2g(p2g, particles, (int64_t)nx * ny * nz, pool_bricks > 0);
    VF_REQUIRE(pool_bricks == 0 || (p2g == VF_P2G_TILE && !(flags & (VF_NO_SORT | VF_TENSION))), VF_EINVAL,
               "sparse storage runs the sorted tiled schedule without tension");
    VF_REQUIRE(pool_bricks >= 0, VF_EINVAL, "a pool needs bricks, got %d", pool_bricks);
    int32_t rc = require_device();
    if (rc) return rc;
    vf_mpm3* h = new vf_mpm3();
    h->nx = nx;
    h->ny = ny;
    h->nz = nz;
    h->np = particles;
    h->flags = flags;
    h->p2g = p2g;
    h->sort = !(flags & VF_NO_SORT);
    h->d.nx = nx;
    h->d.ny = ny;
    h->d.nz = nz;
    h->d.nbx = (nx - 2 + BRICK - 1) / BRICK;
    h->d.nby = (ny - 2 + BRICK - 1) / BRICK;
    h->d.nbz = (nz - 2 + BRICK - 1) / BRICK;
    h->nbricks = h->d.nbx * h->d.nby * h->d.nbz;
    h->nkeys = (int64_t)h->nbricks * 512;
    h->nodes = (int64_t)nx * ny * nz;
    h->stride = ((int64_t)particles + 63) / 64 * 64;
    h->sparse = pool_bricks > 0;
    h->pnx = (nx + POOL_BRICK - 1) / POOL_BRICK;
    h->pny = (ny + POOL_BRICK - 1) / POOL_BRICK;
    h->pnz = (nz + POOL_BRICK - 1) / POOL_BRICK;
    h->npages = h->pnx * h->pny * h->pnz;
    h->pool_cap = h->sparse ? std::min(pool_bricks, h->npages) : 0;
    const size_t grid_bytes = h->sparse ? (size_t)h->pool_cap * POOL_NODES * 16 : (size_t)h->nodes * 16;
    auto fail = [&](int32_t code) {
        delete h;
        return code;
    };
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        set_error("cudaStreamCreate failed");
        return fail(VF_ECUDA);
    }
    size_t pbytes = (size_t)h->stride * NF3 * sizeof(float);
    if ((rc = h->part[0].alloc(pbytes)) || (rc = h->part[1].alloc(pbytes)) ||
        (rc = h->key.alloc((size_t)particles * 4)) || (rc = h->cursor.alloc((size_t)h->nkeys * 4)) ||
        (rc = h->perm.alloc((size_t)particles * 4)) || (rc = h->cell_count.alloc((size_t)h->nkeys * 4)) ||
        (rc = h->cell_start.alloc((size_t)(h->nkeys + 1) * 4)) ||
        (rc = h->brick_count.alloc((size_t)h->nbricks * 4)) ||
        (rc = h->brick_start.alloc((size_t)(h->nbricks + 1) * 4)) ||
        (rc = h->active[0].alloc((size_t)h->nbricks * 4)) || (rc = h->active[1].alloc((size_t)h->nbricks * 4)) ||
        (rc = h->n_active.alloc(4 * sizeof(int))) || (rc = h->grid[0].alloc(grid_bytes)) ||
        (rc = h->grid[1].alloc(grid_bytes)) || (!h->sparse && (rc = h->vel.alloc((size_t)h->nodes * 16))) ||
        (rc = h->params.alloc(sizeof(Params3))) || (rc = h->status.alloc(64)) || (rc = h->scratch.alloc(64)) ||
        (rc = h->nominal.alloc(16)))
        return fail(rc);
    if (h->sparse && ((rc = h->page[0].alloc((size_t)h->npages * 4)) || (rc = h->page[1].alloc((size_t)h->npages * 4)) ||
                      (rc = h->mark.alloc((size_t)h->npages * 4)) || (rc = h->n_used.alloc(2 * sizeof(int)))))
        return fail(rc);
    h->tension = (flags & VF_TENSION) != 0;
    h->fused = h->fuse_wanted && fuse_applies(h);
    if (h->tension && ((rc = h->colour[0].alloc((size_t)h->nodes * 4)) || (rc = h->colour[1].alloc((size_t)h->nodes * 4)) ||
                       (rc = h->stress.alloc((size_t)6 * h->nodes * 4))))
        return fail(rc);
    if (fused_prepare() != cudaSuccess) {
        set_error("cannot give the fused step its shared memory");
        return fail(VF_ECUDA);
    }
    if (p2g_tile_prepare() != cudaSuccess) {
        set_error("cannot give the tiled scatter %zu bytes of shared memory", p2g_tile_smem());
        return fail(VF_ECUDA);
    }
    vf_mpm3_prepared* p = new vf_mpm3_prepared();
    p->sim = h;
    *out = p;
    return VF_OK;
}

}  // namespace

extern "C" {

int32_t vf_mpm3_prepare(int32_t nx, int32_t ny, int32_t nz, int32_t particles, uint32_t flags,
                        vf_mpm3_prepared** out) {
    return prepare3(nx, ny, nz, particles, flags, 0, out);
}

int32_t vf_mpm3_prepare_sparse(int32_t nx, int32_t ny, int32_t nz, int32_t particles, uint32_t flags,
                               int32_t pool_bricks, vf_mpm3_prepared** out) {
    VF_REQUIRE(pool_bricks >= 1, VF_EINVAL, "a sparse grid needs a pool of at least one brick, got %d", pool_bricks);
    return prepare3(nx, ny, nz, particles, flags, pool_bricks, out);
}

int32_t vf_mpm3_pool_used(vf_mpm3* h, int32_t* used) {
    VF_REQUIRE(h && used, VF_EINVAL, "null argument");
    VF_REQUIRE(h->sparse, VF_ESTATE, "this simulation's grid is dense");
    VF_TRY_CUDA(cudaMemcpyAsync(used, h->n_used.as<int>() + h->grid_last, 4, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return check_status(h);
}

int32_t vf_mpm3_pool_capacity(const vf_mpm3* h) { return h ? h->pool_cap : 0; }

void vf_mpm3_prepared_close(vf_mpm3_prepared* p) {
    if (!p) return;
    if (!p->taken && p->sim) {
        vf_mpm3_destroy(p->sim);
    }
    p->sim = nullptr;
    p->taken = true;
    delete p;
}

int32_t vf_mpm3_create(vf_mpm3_prepared* p, vf_mpm3** out) {
    VF_REQUIRE(p && out, VF_EINVAL, "null argument");
    VF_REQUIRE(!p->taken && p->sim, VF_ESTATE, "this preparation has already been made a simulation, or closed");
    vf_mpm3* h = p->sim;
    p->taken = true;
    p->sim = nullptr;
    delete p;
    // ParticleSimulation3(Prepared) clears every buffer (runner.clear(), ParticleSimulation3.java:189)
    for (DeviceBuffer* b : {&h->part[0], &h->part[1], &h->key, &h->cursor, &h->perm, &h->cell_count, &h->cell_start,
                            &h->brick_count, &h->brick_start, &h->active[0], &h->active[1], &h->n_active,
                            &h->grid[0], &h->grid[1], &h->vel, &h->params, &h->status, &h->scratch, &h->mark,
                            &h->n_used}) {
        if (b->ptr && cudaMemsetAsync(b->ptr, 0, b->bytes, h->stream) != cudaSuccess) {
            set_error("clearing buffers failed");
            vf_mpm3_destroy(h);
            return VF_ECUDA;
        }
    }
    for (DeviceBuffer* b : {&h->page[0], &h->page[1]}) {
        if (b->ptr && cudaMemsetAsync(b->ptr, 0xff, b->bytes, h->stream) != cudaSuccess) {   // no brick has a slot
            set_error("clearing buffers failed");
            vf_mpm3_destroy(h);
            return VF_ECUDA;
        }
    }
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
        set_error("clearing buffers failed");
        vf_mpm3_destroy(h);
        return VF_ECUDA;
    }
    *out = h;
    return VF_OK;
}

int32_t vf_mpm3_load(vf_mpm3* h, const float* x, const float* y, const float* z, const float* u, const float* v,
                     const float* w, const float* m, const int32_t* params, int32_t nparams) {
    VF_REQUIRE(h && x && y && z && u && v && w && m, VF_EINVAL, "null argument");
    drop_ahead(h);
    int32_t rc = upload_params(h, params, nparams);
    if (rc) return rc;
    float* base = h->part[h->cur].as<float>();
    const float* src[7] = {x, y, z, u, v, w, m};
    for (int f = 0; f < 7; f++)
        VF_TRY_CUDA(cudaMemcpyAsync(base + f * h->stride, src[f], (size_t)h->np * 4, cudaMemcpyHostToDevice, h->stream));
    VF_TRY_CUDA(fill_f32(base + J * h->stride, h->np, 1.0f, h->stream));
    VF_TRY_CUDA(cudaMemsetAsync(base + C00 * h->stride, 0, (size_t)9 * h->stride * 4, h->stream));
    if ((rc = measure_nominal(h))) return rc;
    rc = reset_counts(h);
    if (rc) return rc;
    VF_TRY_CUDA(cudaMemsetAsync(h->grid[0].ptr, 0, h->grid[0].bytes, h->stream));
    VF_TRY_CUDA(cudaMemsetAsync(h->grid[1].ptr, 0, h->grid[1].bytes, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    h->grid_dirty[0] = h->grid_dirty[1] = 0;
    h->view_fresh = false;
    h->steps = 0;
    h->loaded = true;
    return VF_OK;
}

int32_t vf_mpm3_params(vf_mpm3* h, const int32_t* params, int32_t nparams) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    drop_ahead(h);   // the scatter made ahead used the old params
    return upload_params(h, params, nparams);
}

int32_t vf_mpm3_advance(vf_mpm3* h, int32_t count) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    VF_REQUIRE(count >= 0, VF_EINVAL, "count must be >= 0, got %d", count);
    uint64_t seen[2] = {0, 0};   // the state before each of the last two steps
    for (int k = 0; k < count;) {
        const uint64_t sig = step_sig(h);
        if (h->use_graph && !h->prof.on && count - k >= 2) {
            if (h->pair && h->pair_sig == sig) {
                // the pair leaves the state it started from; only the counters move
                VF_TRY_CUDA(cudaGraphLaunch(h->pair, h->stream));
                h->passes_run += 2;
                h->prof.launches += h->pair_launches;
                h->view_fresh = false;
                h->steps += 2;
                k += 2;
                continue;
            }
            if (sig == seen[1] && (h->p2g != VF_P2G_FIXED || h->fixed.ptr)) {
                if (capture_pair(h, sig) == VF_OK) {
                    h->steps += 2;
                    k += 2;
                    continue;
                }
                h->use_graph = false;   // this handle's steps do not capture; they run as launches
            }
        }
        int32_t rc = step_once(h);
        if (rc) return rc;
        h->steps++;
        k++;
        seen[1] = seen[0];
        seen[0] = sig;
    }
    return VF_OK;
}

int32_t vf_mpm3_set_graph(vf_mpm3* h, int32_t on) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    h->use_graph = on != 0;
    return VF_OK;
}

int32_t vf_mpm3_run(vf_mpm3* h, uint32_t passes) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    drop_ahead(h);
    int32_t rc = run_passes(h, passes, false);
    if (rc) return rc;
    return check_status(h);
}

int32_t vf_mpm3_read(vf_mpm3* h, int32_t field, float* out, int64_t n) {
    VF_REQUIRE(h && out, VF_EINVAL, "null argument");
    if (field >= VF3_GM && field <= VF3_GW) {
        VF_REQUIRE(n == h->nodes, VF_EINVAL, "grid fields hold %lld floats, got %lld", (long long)h->nodes, (long long)n);
        float4* last;
        int32_t rc = last_grid(h, &last);
        if (rc) return rc;
        const float4* src = last;
        int comp = field - VF3_GM;
        if (field >= VF3_GU) {
            Step3 s = make_step(h);
            if (h->sparse) {
                // the grid update over the unpacked box (sparse storage has no tension)
                if (!h->vel.ptr && (rc = h->vel.alloc((size_t)h->nodes * 16))) return rc;
                s.grid = last;
                s.vel = h->vel.as<float4>();
                VF_LAUNCH(h->prof, "k_grid3_dense", h->stream, k_grid3_dense, div_up(h->nodes, 256), 256, 0, s);
            } else if ((rc = grid_pass(h, s, ref_grid(h)))) {
                return rc;
            }
            src = h->vel.as<float4>();
            comp = field - VF3_GU;
        }
        float* tmp = nullptr;
        VF_TRY_CUDA(cudaMallocAsync((void**)&tmp, (size_t)h->nodes * 4, h->stream));
        k_unpack_grid3<<<div_up(h->nodes, 256), 256, 0, h->stream>>>(src, tmp, h->nodes, comp);
        VF_CHECK_LAUNCH();
        VF_TRY_CUDA(cudaMemcpyAsync(out, tmp, (size_t)h->nodes * 4, cudaMemcpyDeviceToHost, h->stream));
        VF_TRY_CUDA(cudaFreeAsync(tmp, h->stream));
        VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
        return check_status(h);
    }
    float* ptr;
    int64_t len;
    int32_t rc = field_pointer(h, field, &ptr, &len);
    if (rc) return rc;
    VF_REQUIRE(n == len, VF_EINVAL, "particle fields hold %lld floats, got %lld", (long long)len, (long long)n);
    VF_TRY_CUDA(cudaMemcpyAsync(out, ptr, (size_t)len * 4, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return check_status(h);
}

int32_t vf_mpm3_write(vf_mpm3* h, int32_t field, const float* in, int64_t n) {
    VF_REQUIRE(h && in, VF_EINVAL, "null argument");
    float* ptr;
    int64_t len;
    int32_t rc = field_pointer(h, field, &ptr, &len);
    if (rc) return rc;
    VF_REQUIRE(n == len, VF_EINVAL, "particle fields hold %lld floats, got %lld", (long long)len, (long long)n);
    drop_ahead(h);
    VF_TRY_CUDA(cudaMemcpyAsync(ptr, in, (size_t)len * 4, cudaMemcpyHostToDevice, h->stream));
    if (field <= VF3_Z && h->counted) {
        rc = reset_counts(h);
        if (rc) return rc;
    }
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return VF_OK;
}

int64_t vf_mpm3_key_count(const vf_mpm3* h) { return h ? h->nkeys : 0; }

int32_t vf_mpm3_read_starts(vf_mpm3* h, int32_t* out, int64_t n) {
    VF_REQUIRE(h && out, VF_EINVAL, "null argument");
    VF_REQUIRE(n == h->nkeys + 1, VF_EINVAL, "starts hold %lld words", (long long)(h->nkeys + 1));
    VF_REQUIRE(h->sorted_valid, VF_ESTATE, "no sort has run");
    int* tmp = nullptr;
    VF_TRY_CUDA(cudaMallocAsync((void**)&tmp, (size_t)n * 4, h->stream));
    k_dense_starts3<<<div_up(n, 256), 256, 0, h->stream>>>(h->cell_start.as<int>(), h->brick_start.as<int>(), tmp,
                                                            h->nkeys, h->np);
    VF_CHECK_LAUNCH();
    VF_TRY_CUDA(cudaMemcpyAsync(out, tmp, (size_t)n * 4, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaFreeAsync(tmp, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return VF_OK;
}

int32_t vf_mpm3_finish(vf_mpm3* h) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return check_status(h);
}

int32_t vf_mpm3_device_ptr(vf_mpm3* h, const char* name, void** ptr, int32_t* stride) {
    VF_REQUIRE(h && name && ptr && stride, VF_EINVAL, "null argument");
    static const char* grid_names[4] = {"gm", "gmu", "gmv", "gmw"};
    for (int k = 0; k < 4; k++)
        if (!strcmp(name, grid_names[k])) {
            float4* last;
            int32_t rc = last_grid(h, &last);
            if (rc) return rc;
            *ptr = reinterpret_cast<float*>(last) + k;
            *stride = 4;
            return VF_OK;
        }
    static const char* part_names[3] = {"x", "y", "z"};
    for (int k = 0; k < 3; k++)
        if (!strcmp(name, part_names[k])) {
            *ptr = h->part[h->cur].as<float>() + (int64_t)k * h->stride;
            *stride = 1;
            return VF_OK;
        }
    set_error("no buffer named '%s'; it has gm, gmu, gmv, gmw, x, y, z", name);
    return VF_EINVAL;
}

void* vf_mpm3_stream(vf_mpm3* h) { return h ? (void*)h->stream : nullptr; }

int32_t vf_mpm3_read_fixed(vf_mpm3* h, int32_t field, int64_t* out, int64_t n) {
    VF_REQUIRE(h && out, VF_EINVAL, "null argument");
    VF_REQUIRE(field >= 0 && field < 4, VF_EINVAL, "the exact grid has fields 0..3 (m, mu, mv, mw), got %d", field);
    VF_REQUIRE(n == h->nodes, VF_EINVAL, "the exact grid has %lld nodes, got %lld", (long long)h->nodes, (long long)n);
    VF_REQUIRE(h->fixed_valid, VF_ESTATE, "the last scatter did not run the exact schedule (VF_P2G_FIXED)");
    VF_TRY_CUDA(cudaMemcpyAsync(out, h->fixed.as<long long>() + (int64_t)field * h->nodes, (size_t)n * 8,
                                cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return check_status(h);
}

int32_t vf_mpm3_set_p2g(vf_mpm3* h, int32_t schedule) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    VF_REQUIRE(schedule >= VF_P2G_TILE && schedule <= VF_P2G_AUTO, VF_EINVAL, "no scatter schedule %d", schedule);
    schedule = resolve_p2g(schedule, h->np, h->nodes, h->sparse);
    VF_REQUIRE(!h->sparse || schedule == VF_P2G_TILE, VF_EINVAL, "sparse storage runs the tiled schedule only");
    if (schedule == VF_P2G_TILE && h->p2g != VF_P2G_TILE) {
        // the dense pipeline leaves both grids dense-dirty
        for (int g = 0; g < 2; g++)
            if (h->grid_dirty[g]) h->grid_dirty[g] = 2;
    }
    drop_ahead(h);
    h->p2g = schedule;
    h->fused = h->fuse_wanted && fuse_applies(h);
    return VF_OK;
}

int32_t vf_mpm3_set_fused(vf_mpm3* h, int32_t on) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    drop_ahead(h);
    h->fuse_wanted = on != 0;
    h->fused = h->fuse_wanted && fuse_applies(h);
    return VF_OK;
}

int32_t vf_mpm3_fused(const vf_mpm3* h) { return h && h->fused ? 1 : 0; }

int32_t vf_mpm3_schedule(const vf_mpm3* h) { return h ? h->p2g : -1; }

int32_t vf_mpm3_nominal_mass(vf_mpm3* h, float* out) {
    VF_REQUIRE(h && out, VF_EINVAL, "null argument");
    VF_TRY_CUDA(cudaMemcpyAsync(out, h->nominal.ptr, 4, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return VF_OK;
}

int32_t vf_mpm3_touched_nodes(vf_mpm3* h, int64_t* out) {
    VF_REQUIRE(h && out, VF_EINVAL, "null argument");
    unsigned long long* c = h->scratch.as<unsigned long long>();
    VF_TRY_CUDA(cudaMemsetAsync(c, 0, 8, h->stream));
    float4* last;
    int32_t rc = last_grid(h, &last);
    if (rc) return rc;
    k_touched3<<<div_up(h->nodes, 256), 256, 0, h->stream>>>(last, h->nodes, c);
    VF_CHECK_LAUNCH();
    unsigned long long v = 0;
    VF_TRY_CUDA(cudaMemcpyAsync(&v, c, 8, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    *out = (int64_t)v;
    return VF_OK;
}

// ParticleDiagnostics.of (ParticleDiagnostics.java:126-148) over the device-resident J: the reference
// reads J back and reduces on the host; so does this (percentiles need the sorted values).
int32_t vf_mpm3_particle_diagnostics(vf_mpm3* h, double speed, double sound, double dt, double out[7]) {
    VF_REQUIRE(h && out, VF_EINVAL, "null argument");
    if (!h->pdiag.ptr) {
        int32_t rc = h->pdiag.alloc(pdiag_scratch_bytes());
        if (rc) return rc;
    }
    unsigned r[5];
    int32_t rc = pdiag_run(h->part[h->cur].as<float>() + (int64_t)J * h->stride, h->np, h->pdiag.ptr, h->stream, r);
    if (rc) return rc;
    const int64_t n = r[0];
    out[4] = speed / sound;
    out[5] = (speed + sound) * dt;
    out[6] = (double)(h->np - n);
    if (n == 0) {
        out[0] = out[1] = out[2] = out[3] = 0;
        return VF_OK;
    }
    // Java's 1 / valid[k] on a float[] is a float division; the record's double holds the float quotient
    out[0] = (double)(1.0f / bits_to_float((int32_t)r[2]));
    out[1] = (double)(1.0f / bits_to_float((int32_t)r[1]));
    out[2] = (double)(1.0f / bits_to_float((int32_t)r[3]));
    out[3] = (double)(1.0f / bits_to_float((int32_t)r[4]));
    return VF_OK;
}

int64_t vf_mpm3_steps(const vf_mpm3* h) { return h ? h->steps : 0; }

int32_t vf_mpm3_profile(vf_mpm3* h, int32_t enable) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    h->prof.reset();
    h->prof.on = enable != 0;
    return VF_OK;
}

int32_t vf_mpm3_profile_read(vf_mpm3* h, int32_t index, char* name, size_t cap, double* total_ms, int64_t* launches) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    return h->prof.read(index, name, cap, total_ms, launches);
}

int64_t vf_mpm3_launches(const vf_mpm3* h) { return h ? h->prof.launches : 0; }

int32_t vf_mpm3_on_gpu(const vf_mpm3* h) { return h ? 1 : 0; }

int32_t vf_mpm3_snapshot(vf_mpm3* h, void* buf, int64_t cap, int64_t* size) {
    VF_REQUIRE(h && size, VF_EINVAL, "null argument");
    const size_t fields = (size_t)NF3 * h->np * 4, grid = (size_t)h->nodes * 16;
    const uint64_t payload = SNAP3_WORDS * 4 + fields + grid;
    *size = (int64_t)(sizeof(SnapHeader) + payload);
    if (!buf) return VF_OK;
    VF_REQUIRE(cap >= *size, VF_EINVAL, "a snapshot of this simulation takes %lld bytes, the buffer has %lld",
               (long long)*size, (long long)cap);
    VF_REQUIRE(h->loaded, VF_ESTATE, "nothing loaded");
    char* body = static_cast<char*>(buf) + sizeof(SnapHeader);
    int32_t words[SNAP3_WORDS] = {0};
    const Params3& p = h->hparams;
    const float w[7] = {p.dt, p.gx, p.gy, p.gz, p.bulk, p.rho0, p.sigma};
    memcpy(words, w, sizeof w);
    memcpy(body, words, sizeof words);
    const float* base = h->part[h->cur].as<float>();
    char* dst = body + sizeof words;
    for (int f = 0; f < NF3; f++)
        VF_TRY_CUDA(cudaMemcpyAsync(dst + (size_t)f * h->np * 4, base + f * h->stride, (size_t)h->np * 4,
                                    cudaMemcpyDeviceToHost, h->stream));
    float4* last;
    int32_t rc0 = last_grid(h, &last);
    if (rc0) return rc0;
    VF_TRY_CUDA(cudaMemcpyAsync(dst + fields, last, grid, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    int32_t rc = check_status(h);
    if (rc) return rc;
    SnapHeader hd = snap_header(SNAP_MPM3, h->nx, h->ny, h->nz, (int32_t)(h->flags & SNAP3_FLAGS), h->np, h->steps,
                                payload);
    hd.checksum = fnv1a(body, payload);
    memcpy(buf, &hd, sizeof hd);
    return VF_OK;
}

int32_t vf_mpm3_restore(vf_mpm3* h, const void* buf, int64_t size) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    const size_t fields = (size_t)NF3 * h->np * 4, grid = (size_t)h->nodes * 16;
    SnapHeader want = snap_header(SNAP_MPM3, h->nx, h->ny, h->nz, (int32_t)(h->flags & SNAP3_FLAGS), h->np, 0,
                                  SNAP3_WORDS * 4 + fields + grid);
    SnapHeader got;
    int32_t rc = snap_check(buf, size, want, &got);
    if (rc) return rc;
    drop_ahead(h);
    const char* body = static_cast<const char*>(buf) + sizeof(SnapHeader);
    int32_t words[SNAP3_WORDS];
    memcpy(words, body, sizeof words);
    if ((rc = upload_params(h, words, 7))) return rc;
    float* base = h->part[h->cur].as<float>();
    const char* src = body + sizeof words;
    for (int f = 0; f < NF3; f++)
        VF_TRY_CUDA(cudaMemcpyAsync(base + f * h->stride, src + (size_t)f * h->np * 4, (size_t)h->np * 4,
                                    cudaMemcpyHostToDevice, h->stream));
    if ((rc = measure_nominal(h))) return rc;
    // the last grid goes back where readouts look for it; both buffers are cleared densely before their next scatter
    if (h->sparse) {
        // readouts look in the unpacked box, which holds the snapshot's grid until the next scatter
        if (!h->view.ptr && (rc = h->view.alloc((size_t)h->nodes * 16))) return rc;
        VF_TRY_CUDA(cudaMemcpyAsync(h->view.ptr, src + fields, grid, cudaMemcpyHostToDevice, h->stream));
        h->view_fresh = true;
    } else {
        VF_TRY_CUDA(cudaMemcpyAsync(h->grid[h->grid_last].ptr, src + fields, grid, cudaMemcpyHostToDevice,
                                    h->stream));
    }
    if ((rc = reset_counts(h))) return rc;
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    h->grid_dirty[0] = h->grid_dirty[1] = 2;
    h->sorted_valid = false;
    h->fixed_valid = false;
    h->steps = got.steps;
    h->loaded = true;
    return VF_OK;
}

void vf_mpm3_destroy(vf_mpm3* h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->pair) cudaGraphExecDestroy(h->pair);
    for (DeviceBuffer* b : {&h->part[0], &h->part[1], &h->key, &h->cursor, &h->perm, &h->cell_count, &h->cell_start,
                            &h->brick_count, &h->brick_start, &h->active[0], &h->active[1], &h->n_active,
                            &h->grid[0], &h->grid[1], &h->vel, &h->params, &h->status, &h->scratch})
        b->release();
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

}  // extern "C"
