/*
 * vexfluid.h -- C-ABI of libvexfluid, the B200 (sm_100a) implementation of the
 * data-parallel fluid step of sibarum/vexelray-sim-fluid.
 *
 * It replaces, beneath the reference's three Java runner classes, SupirVast's
 * PassRunner/Accelerator and the IR kernels they run:
 *   ParticleSimulation   (vexelray-sim-fluid-gui/.../gui/ParticleSimulation.java)   -> vf_mpm2_*
 *   ParticleSimulation3  (vexelray-sim-fluid-gui/.../gui/ParticleSimulation3.java)  -> vf_mpm3_*
 *   PatchSimulation      (vexelray-sim-fluid-gui/.../gui/PatchSimulation.java)      -> vf_swe_*
 * The Java classes keep their public methods and call these through Panama FFM
 * downcalls, one per entry point below.
 *
 * Conventions
 *  - Every function returns int32_t status: VF_OK (0) or a negative VF_E* code. The
 *    message of the calling thread's last error is vf_last_error(). Nothing aborts.
 *  - Handles are opaque. The library owns all device memory; host arrays are the
 *    caller's and are copied in and out synchronously.
 *  - Params are the reference's int[] of float bits (Flip.params, Flip3.params,
 *    ShallowWater.params), so Java call sites pass the same arrays.
 *  - Positions in node units; grid index (k*ny + j)*nx + i; SoA f32 particles.
 *  - A handle belongs to the thread that made it (one CUDA stream per handle).
 */
#ifndef VEXFLUID_H
#define VEXFLUID_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
enum {
    VF_OK = 0,
    VF_EINVAL = -1,    /* an argument the reference refuses with IllegalArgumentException */
    VF_ESTATE = -2,    /* a call the object's state or features do not allow (IllegalStateException) */
    VF_ENOMEM = -3,    /* device or host allocation failed */
    VF_ECUDA = -4,     /* a CUDA runtime error; vf_last_error has the text */
    VF_ETIMEOUT = -5,  /* a bounded device-side wait gave up */
    VF_ENODEV = -6,    /* no CUDA device, or not an sm_100 device */
    VF_EDEVICE = -7    /* a kernel set an error bit in the handle's device status word */
};

/* Copies the calling thread's last error message (NUL-terminated, truncated to cap). Returns its length. */
int32_t vf_last_error(char* buf, size_t cap);
/* Library version, and whether a usable CUDA device is present (1) or not (0). */
int32_t vf_version(void);
int32_t vf_device_ok(void);
/* The architecture the library's kernels were compiled for, as the runtime reports it for one of them
 * (cudaFuncAttributes.binaryVersion: 100 for sm_100a code). VF_ENODEV without a device. */
int32_t vf_binary_version(int32_t* out);
/* Selects the CUDA device the calling thread's next handles use (one process per GPU). */
int32_t vf_set_device(int32_t device);

/* CUDA events on a handle's stream (vf_*_stream), for a caller timing the device work of its calls. */
int32_t vf_event_create(void** event);
int32_t vf_event_record(void* event, void* stream);
/* Waits for `stop` and returns the device time between the two events. */
int32_t vf_event_elapsed_ms(void* start, void* stop, float* ms);
void vf_event_destroy(void* event);
/* Page-locks (pins) a caller's host range so the synchronous copies of load/read run at full PCIe/C2C
 * speed, and releases it. */
int32_t vf_host_register(void* ptr, size_t bytes);
int32_t vf_host_unregister(void* ptr);

/* ------------------------------------------------------------------ physics flags */
/* Flags for vf_mpm2_create / vf_mpm3_prepare. The reference's physics is the default (0):
 * p = B(1/J - 1) (Flip.java:71-78) and the one-node wall ring (Flip.java:122-131). */
enum {
    VF_EOS_TAIT = 1u << 0,          /* p = k((1/J)^7 - 1), k = the params' bulk word */
    VF_WALL_STICKY_SHIFT = 8,       /* bits 8..15: nodes within this many of an edge are stopped */
    VF_WALL_STICKY_MASK = 0xffu << 8,
    VF_P2G_SHIFT = 16,              /* bits 16..19: the 3D scatter schedule, VF_P2G_* */
    VF_P2G_MASK = 0xfu << 16,
    VF_NO_SORT = 1u << 20,          /* 3D: keep the particles in load order (Flip3Step's behaviour) */
    VF_TENSION = 1u << 21,          /* 3D: surface tension's passes between the scatter and the grid (Flip3Step with
                                       tension, Flip3Step.java:88-109); its strength is sigma, the params' word 6 */
    VF_RELAX = 1u << 22             /* 2D: the advect draws J toward the volume the node mass gives (FlipStep with
                                       relax, Flip.advectRelaxing); the rate is the params' word 11 (Flip.RELAX) */
};
#define VF_WALL_STICKY(t) ((uint32_t)(t) << VF_WALL_STICKY_SHIFT)

/* 3D P2G schedules: the three the 3D config compares. */
enum {
    VF_P2G_TILE = 0,    /* sorted particles, one CTA per 8^3-cell brick, shared-memory window, vector red to HBM */
    VF_P2G_ATOMIC = 1,  /* one thread per particle, 27 vector atomics (Flip3.java:225-243's direct scatter) */
    VF_P2G_WARP = 2,    /* one thread per particle, runs of one cell summed across the warp first
                           (Scatter.segmentedDeposit, Scatter.java:385-439, over 27 nodes x 4 fields) */
    VF_P2G_FIXED = 3,   /* exact: every node amount quantized to 2^-40 and added with 64-bit integer atomics, so the
                           grid is the same to the bit in any order and its total mass is the particles' quantized
                           masses' sum exactly (the 3D form of FixedScatter.java:24-60, with 64-bit sums) */
    VF_P2G_AUTO = 4     /* the schedule measured fastest for the handle's size, chosen once at creation (or by
                           vf_mpm3_set_p2g): warp-aggregated below 600k particles on grids under 2^22 nodes, where
                           the tile's one warp per unit of cells leaves much of the GPU idle (1.8x at 17k
                           particles), the tile otherwise and always with sparse storage. The scenes of the
                           reference's scale (32 to 96 nodes a side) take the warp-aggregated scatter */
};

/* ------------------------------------------------------------------ 2D particles (ParticleSimulation) */
typedef struct vf_mpm2 vf_mpm2;

enum {   /* fields for vf_mpm2_read / vf_mpm2_write (FlipStep.java:95-110 buffer names) */
    VF2_X = 0, VF2_Y, VF2_U, VF2_V, VF2_M, VF2_J, VF2_C00, VF2_C01, VF2_C10, VF2_C11,
    VF2_GM = 16, VF2_GMU, VF2_GMV, VF2_GU, VF2_GV
};

/* new ParticleSimulation(nx, ny, particles) (ParticleSimulation.java:39-81): nx, ny >= 3
 * (Scatter.java:516-520 needs >= 2; the quadratic stencil needs 3), particles >= 1 (FlipStep.java:86-88).
 * flags: VF_EOS_TAIT, VF_WALL_STICKY(t), VF_RELAX (ParticleSimulation(..., relax)). The sort's counts start at
 * zero. */
int32_t vf_mpm2_create(int32_t nx, int32_t ny, int32_t particles, uint32_t flags, vf_mpm2** out);
/* ParticleSimulation.load (ParticleSimulation.java:129-143): positions, velocities and masses; J = 1, C = 0;
 * params = Flip.params words (>= 5); resets the step count. */
int32_t vf_mpm2_load(vf_mpm2* h, const float* x, const float* y, const float* u, const float* v, const float* m,
                     const int32_t* params, int32_t nparams);
/* ParticleSimulation.params(int[]) (ParticleSimulation.java:170-172) */
int32_t vf_mpm2_params(vf_mpm2* h, const int32_t* params, int32_t nparams);
/* ParticleSimulation.advance(count, sortEvery) (ParticleSimulation.java:175-183): sorts first on every step
 * whose number (counted across calls) is a multiple of sort_every (>= 1). */
int32_t vf_mpm2_advance(vf_mpm2* h, int32_t count, int32_t sort_every);
/* advance's steps replayed from CUDA graphs, a sort and the sort_every steps after it per graph launch (one graph
 * for each of the two particle sets a sort leaves current, captured on first use); steps that do not fill such a
 * block are launched one by one. Results are those of the launched steps. Off by default; no counterpart in the
 * reference. */
int32_t vf_mpm2_set_graph(vf_mpm2* h, int32_t on);
/* One FlipStep.step() (clear, scatter, grid, advect), and one FlipStep.sort(), without counting a step:
 * what the reference's test Rig runs (Rig.java:30-34). */
int32_t vf_mpm2_step(vf_mpm2* h);
int32_t vf_mpm2_sort(vf_mpm2* h);
/* Readbacks (grid(), positions(), velocities(), masses(), compression(); ParticleSimulation.java:190-220)
 * and writes (compression(float[]) at 213-215; any particle field for tests). n must equal the field's length. */
int32_t vf_mpm2_read(vf_mpm2* h, int32_t field, float* out, int64_t n);
int32_t vf_mpm2_write(vf_mpm2* h, int32_t field, const float* in, int64_t n);
/* The last sort's cell starts, (nx-1)(ny-1)+1 words (Scatter.cellStarts' layout, Scatter.java:484-502). */
int32_t vf_mpm2_read_starts(vf_mpm2* h, int32_t* out, int64_t n);
int64_t vf_mpm2_steps(const vf_mpm2* h);
int32_t vf_mpm2_on_gpu(const vf_mpm2* h);
void vf_mpm2_destroy(vf_mpm2* h);

/* ------------------------------------------------------------------ 2D bilinear P2G (Scatter) */
/* Scatter.Mode (Scatter.java:122-144): the four schedules of the bilinear transfer. */
enum { VF_SCATTER_GRID = 0, VF_SCATTER_PRE_REDUCED = 1, VF_SCATTER_GATHER = 2, VF_SCATTER_SEGMENTED = 3 };
/* One bilinear P2G of host particles onto an nx x ny grid (Scatter.kernel/preReduced/gather/segmented,
 * Scatter.java:154-350); GATHER needs the particles in cell order (Scatter.cellStarts refuses others:
 * VF_EINVAL). Outputs gm, gmu, gmv of nx*ny floats. */
int32_t vf_scatter2(int32_t mode, int32_t nx, int32_t ny, const float* x, const float* y, const float* u,
                    const float* v, const float* m, int64_t np, float* gm, float* gmu, float* gmv);
/* The fixed-point bilinear P2G (FixedScatter.kernel, FixedScatter.java:153-229): i32 registers, the same bits
 * in any order. */
int32_t vf_fixed_scatter2(int32_t nx, int32_t ny, const float* x, const float* y, const float* u, const float* v,
                          const float* m, int64_t np, int32_t mass_bits, int32_t velocity_bits,
                          int32_t* gm, int32_t* gmu, int32_t* gmv);
/* The device sort by cell of host particles (SortTest.Sorter: Scatter.sortCount + CountingSort,
 * SortTest.java:255-313), stable: writes the permutation (perm[d] = source index) and the starts. */
int32_t vf_sort2(int32_t nx, int32_t ny, const float* x, const float* y, int64_t np, int32_t* perm,
                 int32_t* starts);
/* vf_sort2 without any device allocation. No counterpart in the reference: it is for callers that must
 * not allocate device memory while they run -- a host that budgets all device memory up front, or a
 * real-time loop where cudaMalloc/cudaFree would synchronise the device and stall the frame. Its scratch
 * is one fixed array in the library (about 7 MB, held on every GPU that loads the library until exit), so
 * it takes at most 262144 particles and 262144 cells ((nx-1)(ny-1)); larger inputs get VF_EINVAL. Every
 * call shares that array: calls that overlap on the GPU race, so a caller with several threads or streams
 * serialises them. Each call looks up the array's device address on the current device; the first call on a
 * device also loads the library there, so make it before any stream capture. Same outputs as vf_sort2. */
int32_t vf_sort2_noalloc(int32_t nx, int32_t ny, const float* x, const float* y, int64_t np, int32_t* perm,
                         int32_t* starts);

/* ------------------------------------------------------------------ batched 2D scenes */
/* Many independent 2D scenes (each a ParticleSimulation's FlipStep: sort by cell, scatter, grid, advect)
 * stepped together: one cooperative persistent kernel launch per step over every scene, with CUDA graphs
 * replaying the launches. No counterpart in the reference. Scenes of one batch share the physics flags
 * (VF_EOS_TAIT, VF_WALL_STICKY(t)); each has its own grid, particle count and Flip.params words. */
typedef struct vf_mpm2_batch vf_mpm2_batch;

typedef struct {
    int32_t nx, ny;          /* grid nodes, >= 3 each */
    int32_t particles;       /* >= 1 */
    int32_t tile_x, tile_y;  /* P2G/G2P tile in stencil cells: one of the VF_BATCH_TILES shapes (0, 0 = 16 x 16) */
    int32_t params[5];       /* Flip.params words [dt, gx, gy, bulk, rho0] (Flip.java:145-211) */
} vf_scene2;

/* The tile shapes a scene may use (x, y pairs), and the block sizes a batch may launch with. */
#define VF_BATCH_TILES {{8, 8}, {16, 8}, {16, 16}, {32, 8}, {32, 16}}
#define VF_BATCH_BLOCKS {128, 256, 512}

/* Builds a batch: scenes are copied; block is the CTA size (one of VF_BATCH_BLOCKS, 0 = 256). */
int32_t vf_mpm2_batch_create(const vf_scene2* scenes, int32_t nscenes, uint32_t flags, int32_t block,
                             vf_mpm2_batch** out);
/* Loads every scene's particles: each array holds the scenes' particles one scene after another (sum of
 * particles floats). J = 1, C = 0; the step count restarts at zero. */
int32_t vf_mpm2_batch_load(vf_mpm2_batch* h, const float* x, const float* y, const float* u, const float* v,
                           const float* m);
/* count steps of every scene (FlipStep.step with a sort every step), submitted as CUDA graph replays.
 * Returns when submitted; vf_mpm2_batch_finish waits and reports device errors. */
int32_t vf_mpm2_batch_advance(vf_mpm2_batch* h, int32_t count);
int32_t vf_mpm2_batch_finish(vf_mpm2_batch* h);
/* The polls a CTA of the step kernel makes at a grid barrier before it gives up (0, the default, is about a
 * second's worth). A barrier that gives up sets the device status: the step's kernel ends, the next blocking call
 * returns VF_ETIMEOUT, and the batch refuses to step (VF_ESTATE) until it is loaded again, which also restores the
 * default. A test hook for the bounded wait; the reference's analogue is Stepper's runaway guard
 * (vexelray-sim-fluid-core/.../stencil/Stepper.java:88-93). */
int32_t vf_mpm2_batch_set_wait_limit(vf_mpm2_batch* h, int32_t polls);
/* One scene's particle field (VF2_X..VF2_C11, in the batch's sorted order: by tile and cell, the order within a
 * cell unspecified) or the last step's grid
 * (VF2_GM, VF2_GMU, VF2_GMV; nx*ny floats). Blocking. */
int32_t vf_mpm2_batch_read(vf_mpm2_batch* h, int32_t scene, int32_t field, float* out, int64_t n);
/* The tile shape a scene runs with, and the batch's block size and persistent grid size (CTAs). */
int32_t vf_mpm2_batch_config(const vf_mpm2_batch* h, int32_t scene, int32_t* tile_x, int32_t* tile_y,
                             int32_t* block, int32_t* ctas);
/* Device time of the step's five phases (tile scan, cell scan, permute, scatter, gather) summed over the launches
 * since the last call, from the kernel's own clock (%globaltimer at every grid barrier), and those launches. */
int32_t vf_mpm2_batch_phases(vf_mpm2_batch* h, double ms[5], int64_t* launches);
int64_t vf_mpm2_batch_particles(const vf_mpm2_batch* h);
int64_t vf_mpm2_batch_steps(const vf_mpm2_batch* h);
int64_t vf_mpm2_batch_launches(const vf_mpm2_batch* h);
void* vf_mpm2_batch_stream(vf_mpm2_batch* h);
void vf_mpm2_batch_destroy(vf_mpm2_batch* h);

/* The tile-shape and block-size autotuner. Each scene is keyed by (particles per occupied cell rounded to a
 * power of two, max(nx, ny) rounded up to a power of two). For every key not found in the JSON cache at
 * cache_path, it times a batch of up to 8 of that key's scenes with each VF_BATCH_TILES shape. It then times
 * the scenes with each VF_BATCH_BLOCKS size, unless the cache holds a block size for this batch's key set.
 * The winners are written to the cache (created if absent; cache_path NULL = no cache). On return, scenes[i]'s
 * tile_x/tile_y and *block hold the choices. Particles are given as for vf_mpm2_batch_load. trials counts the
 * timed configurations (0 when everything came from the cache). */
int32_t vf_mpm2_autotune(vf_scene2* scenes, int32_t nscenes, uint32_t flags, const float* x, const float* y,
                         const float* u, const float* v, const float* m, const char* cache_path, int32_t* block,
                         int32_t* trials);

/* ------------------------------------------------------------------ 3D particles (ParticleSimulation3) */
typedef struct vf_mpm3 vf_mpm3;
typedef struct vf_mpm3_prepared vf_mpm3_prepared;

enum {   /* fields (Flip3.PARTICLE, Flip3.java:112-115; grid names Flip3Step.java:65-67) */
    VF3_X = 0, VF3_Y, VF3_Z, VF3_U, VF3_V, VF3_W, VF3_M, VF3_J,
    VF3_C00, VF3_C01, VF3_C02, VF3_C10, VF3_C11, VF3_C12, VF3_C20, VF3_C21, VF3_C22,
    VF3_GM = 32, VF3_GMU, VF3_GMV, VF3_GMW, VF3_GU, VF3_GV, VF3_GW
};

/* ParticleSimulation3.prepare (ParticleSimulation3.java:110-139): every buffer allocated and every kernel
 * loaded, nothing submitted; may run on any thread. nx, ny, nz >= 3; particles >= 1 (Flip3Step.java:54-56).
 * flags: VF_EOS_TAIT, VF_WALL_STICKY(t), P2G schedule << VF_P2G_SHIFT, VF_NO_SORT, VF_TENSION (prepare(..., tension)).
 * With VF_TENSION the grid readouts VF3_GU..GW include the tension's force. */
int32_t vf_mpm3_prepare(int32_t nx, int32_t ny, int32_t nz, int32_t particles, uint32_t flags,
                        vf_mpm3_prepared** out);
/* As vf_mpm3_prepare, with the grid stored sparsely: no counterpart in the reference, which plans it
 * (docs/sparse-fluid.md:19-62). The nodes live in a pool of pool_bricks bricks of 8^3 nodes (8 KB each, two pools,
 * one per step parity) through a page table over the domain's bricks, rebuilt every step from the bricks the
 * particles' stencils reach; memory for the grid follows the fluid, not the box. The tiled schedule only, sorted,
 * without tension (VF_EINVAL otherwise). A step that needs more bricks than the pool holds skips the nodes of the
 * bricks past it and reports VF_EDEVICE (status bit 8) at the next blocking call. Readouts of the grid unpack the
 * pool into a dense box made on first use. pool_bricks above the domain's brick count is cut to it. */
int32_t vf_mpm3_prepare_sparse(int32_t nx, int32_t ny, int32_t nz, int32_t particles, uint32_t flags,
                               int32_t pool_bricks, vf_mpm3_prepared** out);
/* The bricks the last scatter took from the pool (blocking; VF_ESTATE for a dense grid), and the pool's size. */
int32_t vf_mpm3_pool_used(vf_mpm3* h, int32_t* used);
int32_t vf_mpm3_pool_capacity(const vf_mpm3* h);
/* Prepared.close (ParticleSimulation3.java:94-102): frees a preparation never finished. Idempotent. */
void vf_mpm3_prepared_close(vf_mpm3_prepared* p);
/* new ParticleSimulation3(Prepared) (ParticleSimulation3.java:181-190), on the owning thread: clears the
 * buffers. The preparation is consumed (VF_ESTATE if already taken). */
int32_t vf_mpm3_create(vf_mpm3_prepared* p, vf_mpm3** out);
/* ParticleSimulation3.load (ParticleSimulation3.java:227-275): J = 1, C = 0; params = Flip3.params words (>= 6). */
int32_t vf_mpm3_load(vf_mpm3* h, const float* x, const float* y, const float* z, const float* u, const float* v,
                     const float* w, const float* m, const int32_t* params, int32_t nparams);
int32_t vf_mpm3_params(vf_mpm3* h, const int32_t* params, int32_t nparams);
/* ParticleSimulation3.advance (ParticleSimulation3.java:291-296); with the default flags each step sorts the
 * particles by stencil cell first. */
int32_t vf_mpm3_advance(vf_mpm3* h, int32_t count);
/* advance's steps replayed from a CUDA graph: once the step's host-side state recurs every two steps (after two or
 * three steps), two steps are captured and then replayed, one graph launch per pair, for as long as the state
 * before a pair is the one captured; a change of schedule, a load or a restore is met by a new capture. Results
 * are those of the launched steps. Off by default; no counterpart in the reference, whose runner records each pass
 * into a command buffer. With per-kernel profiling on, steps are launched one by one. */
int32_t vf_mpm3_set_graph(vf_mpm3* h, int32_t on);
/* Passes of one step, for tests (Flip3Test runs clear+scatter alone, Flip3Test.java:90):
 * bit 0 sort, bit 1 clear, bit 2 scatter, bit 3 grid, bit 4 advect. Does not count a step. */
enum { VF3_PASS_SORT = 1, VF3_PASS_CLEAR = 2, VF3_PASS_SCATTER = 4, VF3_PASS_GRID = 8, VF3_PASS_ADVECT = 16 };
int32_t vf_mpm3_run(vf_mpm3* h, uint32_t passes);
/* Readbacks: grid() (ParticleSimulation3.java:302-304; the last scatter's m, mu, mv, mw), velocities(), and
 * any particle field; writes of any particle field. Blocking. */
int32_t vf_mpm3_read(vf_mpm3* h, int32_t field, float* out, int64_t n);
int32_t vf_mpm3_write(vf_mpm3* h, int32_t field, const float* in, int64_t n);
/* The last sort's cell starts over the brick-major stencil-cell keys, vf_mpm3_key_count()+1 words. */
int64_t vf_mpm3_key_count(const vf_mpm3* h);
int32_t vf_mpm3_read_starts(vf_mpm3* h, int32_t* out, int64_t n);
/* ParticleSimulation3.finish (ParticleSimulation3.java:399-402): waits for every step submitted. */
int32_t vf_mpm3_finish(vf_mpm3* h);
/* ParticleSimulation3.vkBuffer(name) (ParticleSimulation3.java:377-383), as a device pointer: "gm", "gmu",
 * "gmv", "gmw" (the last scatter's grid) or "x", "y", "z". *stride is the element stride in floats (4 for the
 * grid, whose nodes are stored as float4 {m, mu, mv, mw}; 1 for particles). Valid until the next step;
 * call vf_mpm3_finish before reading. VF_EINVAL for another name. */
int32_t vf_mpm3_device_ptr(vf_mpm3* h, const char* name, void** ptr, int32_t* stride);
/* The CUDA stream (cudaStream_t) the handle's work is submitted on, for event timing by a caller. */
void* vf_mpm3_stream(vf_mpm3* h);
/* Change the scatter schedule (VF_P2G_*) between steps. */
int32_t vf_mpm3_set_p2g(vf_mpm3* h, int32_t schedule);
/* The fused step, with the sorted tiled schedule on dense storage without tension: a step is the sort and ONE
 * kernel that gathers each particle's velocity and affine matrix from the last grid (Flip3.advect), moves it, and
 * scatters its new state into the next grid (Flip3.scatter of the next step), so a particle's velocity and affine
 * matrix are written once and not read back. The next step's scatter is then made at the end of this one; grid(),
 * the snapshot and the device pointers still show the last step's grid, and anything that changes the particles,
 * the params or the schedule discards the early scatter. Off by default (on = 1 turns it on; 0 runs Flip3Step's
 * passes, the tiled scatter and the tiled gather). No counterpart in the reference. */
int32_t vf_mpm3_set_fused(vf_mpm3* h, int32_t on);
/* 1 when the steps run fused. */
int32_t vf_mpm3_fused(const vf_mpm3* h);
/* The schedule the steps run (VF_P2G_AUTO resolved). */
int32_t vf_mpm3_schedule(const vf_mpm3* h);
/* The smallest positive mass of the last load (or restore), FLT_MAX if none: ParticleSimulation3's nominalMass
 * (ParticleSimulation3.java:248-253), measured on the device during the load; compression() keeps the particles
 * holding at least half of it (ParticleSimulation3.java:312-333). Blocking. */
int32_t vf_mpm3_nominal_mass(vf_mpm3* h, float* out);
/* The last scatter's exact grid when it ran VF_P2G_FIXED (VF_ESTATE otherwise): field 0..3 = m, mu, mv, mw as
 * int64 with 40 fractional bits, n = nx*ny*nz values. No counterpart in the reference. */
int32_t vf_mpm3_read_fixed(vf_mpm3* h, int32_t field, int64_t* out, int64_t n);
/* Nodes with mass after the last scatter (N_t in the roofline's byte count). Blocking. */
int32_t vf_mpm3_touched_nodes(vf_mpm3* h, int64_t* out);
int64_t vf_mpm3_steps(const vf_mpm3* h);
int32_t vf_mpm3_on_gpu(const vf_mpm3* h);
/* A versioned binary snapshot of the simulation, for resume and replay; no counterpart in the reference. The
 * blob: a 64-byte header (magic "VFSNAP", version, kind 3, nx, ny, nz, the physics flags, particles, steps, payload
 * length, FNV-1a 64 of the payload), then 8 param words (7 Flip3.params words and a zero), the 17 particle fields
 * of the current order (x y z u v w m j c00..c22, np floats each) and the last scatter's grid (nodes x float4
 * {m, mu, mv, mw}). buf = null: *size gets the length only. Blocking. restore: the same grid sizes, particle count
 * and physics flags (the scatter schedule and the sort switch may differ), VF_EINVAL on any mismatch or a bad
 * checksum; it sets the step count and leaves the sort to recount. Under VF_P2G_FIXED a restored run continues
 * bit for bit as the original does. */
int32_t vf_mpm3_snapshot(vf_mpm3* h, void* buf, int64_t cap, int64_t* size);
int32_t vf_mpm3_restore(vf_mpm3* h, const void* buf, int64_t size);
/* Kernel accounting: with profiling on, every launch of the handle is bracketed by CUDA events and its
 * device time summed per kernel; profile_read returns entry `index` (VF_EINVAL past the last). launches is
 * the count of kernels the handle has launched since it was made, profiling on or off. */
int32_t vf_mpm3_profile(vf_mpm3* h, int32_t enable);
int32_t vf_mpm3_profile_read(vf_mpm3* h, int32_t index, char* name, size_t cap, double* total_ms, int64_t* launches);
int64_t vf_mpm3_launches(const vf_mpm3* h);
void vf_mpm3_destroy(vf_mpm3* h);

/* ------------------------------------------------------------------ shallow water (PatchSimulation) */
typedef struct vf_swe vf_swe;
enum { VF_EDGE_WALL = 0, VF_EDGE_OPEN = 1 };   /* Edge.java:11-25 */

/* new PatchSimulation(nx, ny, edges) (PatchSimulation.java:58-76); edges = {west, east, south, north}
 * (Edges.java:29). nx, ny >= 1 (ShallowWater.java:167-169). */
int32_t vf_swe_create(int32_t nx, int32_t ny, const int32_t edges[4], vf_swe** out);
/* PatchSimulation.load (PatchSimulation.java:92-109): the state, params = ShallowWater.params words (5);
 * the first step's speed is measured on the host (ShallowWater.fastestWave); the clock restarts at zero. */
int32_t vf_swe_load(vf_swe* h, const float* hcell, const float* hu, const float* hv, const int32_t* params,
                    int32_t nparams);
int32_t vf_swe_params(vf_swe* h, const int32_t* params, int32_t nparams);
/* PatchSimulation.advance(ticks, maxSteps) (PatchSimulation.java:120-145) and its Advance record (33-39). */
int32_t vf_swe_advance(vf_swe* h, int64_t ticks, int32_t max_steps, int32_t* steps, int64_t* spent_ticks,
                       int64_t* behind_ticks);
/* PatchSimulation.read (148-152), fastestWave (158-160), clamped (176-178), now (181-183), steps (186-188). */
int32_t vf_swe_read(vf_swe* h, float* hcell, float* hu, float* hv);
int32_t vf_swe_fastest_wave(vf_swe* h, double* out);
int32_t vf_swe_clamped(vf_swe* h, int32_t* out);
int64_t vf_swe_now(const vf_swe* h);
int64_t vf_swe_steps(const vf_swe* h);
/* The raw rotation, for the reference's test harness (Stepper.java:72-77, 128-130): dispatch n steps
 * k = dispatched, dispatched+1, ... with state k%2 -> (k+1)%2, speed k%3 read / (k+1)%3 max / (k+2)%3 clear,
 * budget k%2 -> (k+1)%2; and the budget words. */
int32_t vf_swe_dispatch(vf_swe* h, int32_t n);
int64_t vf_swe_dispatched(const vf_swe* h);
int32_t vf_swe_write_budget(vf_swe* h, int32_t slot, int32_t ticks);
int32_t vf_swe_read_budget(vf_swe* h, int32_t slot, int32_t* ticks);
/* The exact mode's step kernel: 64 (the default) or 32 stage primitives and fluxes of 64- or 32-cell-wide tiles
 * in shared memory (k_swe_tile, 16 rows); 0 walks columns of 120 x 32-cell strips in registers (k_swe_strip). No
 * counterpart in the reference: results are bit-identical for all three, only the speed differs (the tile measured
 * 0.33 ms a step at 4096^2, the strip walk 0.35). The fast mode (vf_swe_set_exact(h, 0)) always walks strips. */
int32_t vf_swe_set_tile_width(vf_swe* h, int32_t width);
int32_t vf_swe_tile_width(const vf_swe* h);
/* Each step launched as a programmatic dependent of the previous one (its CTAs may become resident during the
 * previous step's last wave and wait on the device for its completion): 1 (the default) or 0 (plain stream
 * order). Bit-identical either way. */
int32_t vf_swe_set_overlap(vf_swe* h, int32_t on);
/* The step's arithmetic. on = 1 (the default): every operation rounded as the reference's strict f32 does, so
 * the state, clock and clamp count equal the reference's CPU step bit for bit. on = 0: the fast mode, the same
 * tile and flux form with fused multiply-adds, one approximate reciprocal of each cell's depth and of each face's
 * wave span, and an approximate wave-speed square root: within a stated tolerance of the reference (about 1e-5
 * relative per cell over tens of steps of smooth flow), the water moving only between neighbours as before. No
 * counterpart in the reference, whose Vulkan path has no correctly rounded division either. */
int32_t vf_swe_set_exact(vf_swe* h, int32_t on);
int32_t vf_swe_exact(const vf_swe* h);
/* A versioned binary snapshot of the patch (kind 2, the same 64-byte header with the edges in flags, 8 bits each):
 * the 16-word device block (speed words in their rotation, budget words, clamp count, params), clock, dispatch
 * count, steps and the last step's ticks (int64 each), then h, hu, hv. Resumes bit for bit, clock included.
 * buf = null: *size gets the length only. restore: VF_EINVAL on another size, edges or a bad checksum. */
int32_t vf_swe_snapshot(vf_swe* h, void* buf, int64_t cap, int64_t* size);
int32_t vf_swe_restore(vf_swe* h, const void* buf, int64_t size);
/* Diagnostics.of(h, hu, hv, g, dry, dt, dx, dy) over the current state (Diagnostics.java:43-81), reduced on the
 * device. out = {volume, minDepth, maxDepth, maxSpeed, maxFroude, maxCourant, nonFinite, negative, wet}. */
int32_t vf_swe_diagnostics(vf_swe* h, double g, double dry, double dt, double dx, double dy, double out[9]);
/* Kernel accounting, as vf_mpm3_profile. */
int32_t vf_swe_profile(vf_swe* h, int32_t enable);
int32_t vf_swe_profile_read(vf_swe* h, int32_t index, char* name, size_t cap, double* total_ms, int64_t* launches);
int64_t vf_swe_launches(const vf_swe* h);
void* vf_swe_stream(vf_swe* h);
int32_t vf_swe_on_gpu(const vf_swe* h);
void vf_swe_destroy(vf_swe* h);

/* The state on the device, for callers that work on it between steps (the learned correction): pointers to
 * the current h, hu, hv (nx*ny floats each, on the handle's stream), valid until the next dispatch. After changing
 * it, vf_swe_measure_speed sets the next step's wave speed from the changed state (as load's fastestWave does). */
int32_t vf_swe_state(vf_swe* h, float** hcell, float** hu, float** hv);
int32_t vf_swe_measure_speed(vf_swe* h);
/* The fine handle's current state averaged over 2x2 blocks into the coarse handle's current state (fine nx, ny
 * = 2 x the coarse's), and the coarse wave speed measured; on the device. */
int32_t vf_swe_restrict(vf_swe* fine, vf_swe* coarse);
/* The inverse for a patch: the coarse cells [x0, x0 + nx/2) x [y0, y0 + ny/2) of `coarse`, each copied to its 2x2
 * fine cells of `fine` (a patch of nx x ny cells), and the fine wave speed measured. */
int32_t vf_swe_prolong(vf_swe* coarse, int32_t x0, int32_t y0, vf_swe* fine);
/* nx x ny coarse cells from (x0, y0) of `coarse` = the means of the fine patch's 2x2 blocks from fine cell
 * (fx0, fy0). */
int32_t vf_swe_restrict_patch(vf_swe* fine, int32_t fx0, int32_t fy0, vf_swe* coarse, int32_t x0, int32_t y0,
                              int32_t nx, int32_t ny);
/* dst's current state = src's (same grid), on the device; dst's wave speed measured. */
int32_t vf_swe_copy_state(vf_swe* dst, vf_swe* src);
/* Per tile of tile x tile cells (row-major, ntiles = ceil(nx/tile) * ceil(ny/tile)): the largest relative depth
 * jump between neighbouring cells, (|dh east| + |dh north|) / max(h, dry), of the current state. */
int32_t vf_swe_jump_indicator(vf_swe* h, int32_t tile, float* out, int32_t ntiles);

/* ------------------------------------------------------------------ the flux-correction network */
/* A 3-layer 5x5 convolutional network (3 -> 32 -> 32 -> 6 channels, ReLU between; bf16 weights and activations,
 * fp32 accumulation on the tensor cores) that corrects a coarse shallow-water state by the divergence of six
 * face fields (the east and north faces' transfer of h, hu, hv; faces on the walls held at zero, so totals are
 * conserved):  U(i,j) -= s_flux (G_e(i,j) - G_e(i-1,j) + G_n(i,j) - G_n(i,j-1)).
 * No counterpart in the reference. Trained on samples (S, P, T): a coarse state S, the plain coarse solver's state
 * P an interval later, and the fine solver's state after that interval restricted to the coarse grid T; the loss
 * is the mean over cells, components and samples of ((P - s_flux Div G(S) - T) / s_res)^2 / 2, and training is
 * Adam on fp32 master parameters. The parameters, in order: w1 [32][25][3], b1 [32], w2 [32][25][32], b2 [32],
 * w3 [6][25][32], b3 [6] (w[cout][ky*5+kx][cin]); the features are (h - 1)*4, hu*4, hv*4. */
typedef struct vf_cnn vf_cnn;

int64_t vf_cnn_param_count(void);
/* For an nx x ny coarse grid: up to `batch` samples per training step, a ring of `samples` sample slots. */
int32_t vf_cnn_create(int32_t nx, int32_t ny, int32_t batch, int32_t samples, float s_flux, float s_res,
                      vf_cnn** out);
/* Reads or writes (write != 0: also resets Adam's moments) the fp32 parameters, vf_cnn_param_count() floats. */
int32_t vf_cnn_params(vf_cnn* h, float* host, int64_t n, int32_t write);
/* Sample slot `slot`, part kind (0 = S, 1 = P, 2 = T): three planes copied in from device (from_host = 0) or host. */
int32_t vf_cnn_put(vf_cnn* h, int32_t slot, int32_t kind, const float* hcell, const float* hu, const float* hv,
                   int32_t from_host);
/* The loss over samples, and (loss_plain non-null) the loss with no correction. */
int32_t vf_cnn_loss(vf_cnn* h, const int32_t* slots, int32_t n, double* loss, double* loss_plain);
/* The loss's gradient (vf_cnn_param_count() floats) over samples, without an update. */
int32_t vf_cnn_gradients(vf_cnn* h, const int32_t* slots, int32_t n, float* grads, double* loss);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on the loss over samples; *loss is the loss before it. */
int32_t vf_cnn_train(vf_cnn* h, const int32_t* slots, int32_t n, float lr, double* loss);
/* The correction: predict from the state at an interval's start (the network's S), apply to the plain solver's
 * state at its end (P); both device planes of the network's grid, e.g. from vf_swe_state. `stream` (a
 * cudaStream_t, e.g. vf_swe_stream) is the stream that produces and consumes the state: the network's work is
 * ordered after that stream's work so far and that stream's later work after the network's, with no host wait;
 * NULL waits on the host instead. vf_cnn_apply without a prediction since the last apply is VF_ESTATE.
 * vf_cnn_correct predicts and applies on one state. */
int32_t vf_cnn_predict(vf_cnn* h, const float* hcell, const float* hu, const float* hv, void* stream);
int32_t vf_cnn_apply(vf_cnn* h, float* hcell, float* hu, float* hv, void* stream);
int32_t vf_cnn_correct(vf_cnn* h, float* hcell, float* hu, float* hv, void* stream);
/* The network's output for sample slot's S: nx*ny*8 floats (six used per cell, the east face's h, hu, hv then the
 * north face's). */
int32_t vf_cnn_fluxes(vf_cnn* h, int32_t slot, float* out);
void* vf_cnn_stream(vf_cnn* h);
/* The forward and input-gradient convolutions' kernels: 0 (the default) tcgen05.mma for every layer (TMA-fed ring
 * of input rows in shared memory, accumulators in tensor memory, warp-specialised); 1 mma.sync with each warp computing several output rows from every A fragment it loads; 2
 * mma.sync with one output row per warp. All compute the same network (to fp32 summation order). The weight
 * gradients always run on mma.sync. */
int32_t vf_cnn_set_path(vf_cnn* h, int32_t path);
/* Waits for the network's stream and reports a kernel's status bits (VF_ETIMEOUT for a bounded wait that expired). */
int32_t vf_cnn_status(vf_cnn* h);
int32_t vf_cnn_profile(vf_cnn* h, int32_t enable);
int32_t vf_cnn_profile_read(vf_cnn* h, int32_t index, char* name, size_t cap, double* total_ms, int64_t* launches);
int64_t vf_cnn_launches(const vf_cnn* h);
void vf_cnn_destroy(vf_cnn* h);

/* ------------------------------------------------------------------ the learned coarse solver */
/* The learned coarse shallow-water solver as one handle; no counterpart in the reference, its error measured
 * against the plain fine solver. An nx x ny coarse patch with walls (cells 2 dx wide) stepped by the plain HLL step; every
 * `interval_ticks` the network `net` (borrowed; NULL: the plain coarse solver) predicts a correction from the
 * interval's start state, on the coarse stream, and it is applied at the interval's end. With `fallback`, tiles
 * of `tile` coarse cells whose relative depth jump (vf_swe_jump_indicator) exceeds `threshold` at an interval's
 * start are stepped by the fine solver instead: the tile and `margin` coarse cells around it, prolonged into a
 * fine patch (open edges inside the domain), stepped through the interval and restricted back. load takes a
 * coarse state with the coarse params (g 9.81, Courant 0.45, dry 1e-6). */
typedef struct vf_swe_learned vf_swe_learned;
int32_t vf_swe_learned_create(int32_t nx, int32_t ny, vf_cnn* net, int64_t interval_ticks, int32_t tile,
                              int32_t fallback, float threshold, int32_t margin, float dx, vf_swe_learned** out);
int32_t vf_swe_learned_load(vf_swe_learned* h, const float* hcell, const float* hu, const float* hv);
/* Intervals until `ticks` are spent (the last one shortened to fit). VF_ESTATE when an interval takes more than
 * 1024 coarse steps (a correction drove the state toward dry or violent flow and the step stopped growing). */
int32_t vf_swe_learned_advance(vf_swe_learned* h, int64_t ticks);
int32_t vf_swe_learned_read(vf_swe_learned* h, float* hcell, float* hu, float* hv);
/* out = {coarse steps, corrections applied, fallback tiles stepped}. */
int32_t vf_swe_learned_counts(const vf_swe_learned* h, int64_t out[3]);
/* The coarse patch, for its readouts (diagnostics, wave speed); owned by the handle. */
vf_swe* vf_swe_learned_coarse(vf_swe_learned* h);
void vf_swe_learned_destroy(vf_swe_learned* h);

/* ------------------------------------------------------------------ particle diagnostics */
/* ParticleDiagnostics.of over a device-resident J (ParticleDiagnostics.java:126-148): out = {minDensity,
 * maxDensity, lowDensity, highDensity, mach, courant, nonFinite}. */
int32_t vf_mpm3_particle_diagnostics(vf_mpm3* h, double speed, double sound, double dt, double out[7]);

#ifdef __cplusplus
}
#endif
#endif /* VEXFLUID_H */
