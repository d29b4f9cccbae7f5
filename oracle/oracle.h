/*
 * oracle.h -- CPU restatement of the reference fluid step, used ONLY as the test
 * oracle and as the timed CPU baseline.
 *
 * This is test infrastructure. Nothing in the product library links, loads or
 * calls it: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * --impl reference legs use it, and only to check results against or as the CPU comparison.
 *
 * The reference (sibarum/vexelray-sim-fluid) is Java that builds SupirVast IR
 * (dev.supirvast:vastir 0.2.3-SNAPSHOT, not vendored, no JDK here), so it cannot
 * run here. Every function below restates one IR kernel expression
 * by expression, in the operand order the IR builds it, in IEEE f32 with no
 * contraction (built -ffp-contract=off), which is what Java's strict float
 * arithmetic computes. Each function cites the reference file:line it follows;
 * paths are relative to vexelray-sim-fluid-core/src/main/java/dev/vexelray/sim/fluid/.
 *
 * Parity pins: the known-answer tests of the reference's own test suite
 * (FlipTest, Flip3Test, ScatterTest, SortTest, ShallowWaterTest,
 * DiagnosticsTest, ParticleDiagnosticsTest) are ported in tests/test_oracle_*.py
 * and run against these functions, with inputs regenerated by a java.util.Random
 * restatement (javarand.c) from the same seeds.
 */
#ifndef VEXFLUID_ORACLE_H
#define VEXFLUID_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- java.util.Random */
/* A restatement of java.util.Random from the Java SE API specification (48-bit LCG,
 * nextFloat/nextDouble/nextInt(bound)/nextGaussian), so the reference tests' seeded
 * inputs (new Random(71), ...) are regenerated bit for bit. */
typedef struct { int64_t seed; int have_next_gaussian; double next_gaussian; } or_jrand;
void   or_jrand_init(or_jrand* r, int64_t seed);
int32_t or_jrand_next(or_jrand* r, int bits);
float  or_jrand_float(or_jrand* r);
double or_jrand_double(or_jrand* r);
int32_t or_jrand_int(or_jrand* r, int32_t bound);
double or_jrand_gaussian(or_jrand* r);
/* n draws of nextFloat into out (a convenience for the Python harness) */
void   or_jrand_floats(or_jrand* r, float* out, int64_t n);

/* ---------------------------------------------------------------- physics options */
/* Equation of state and wall model. REF follows Flip.java / Flip3.java exactly;
 * TAIT and STICKY are the benchmark configurations' physics: p = k((1/J)^7 - 1) with k the bulk word, and
 * every node within `sticky` nodes of an edge stopped. */
enum { OR_EOS_REF = 0, OR_EOS_TAIT = 1 };
typedef struct {
    int eos;          /* OR_EOS_REF: p = B(1/J - 1); OR_EOS_TAIT: p = k((1/J)^7 - 1) */
    int sticky;       /* 0: the reference's wall ring (Flip.java:404-407); t>0: nodes within t of an edge are stopped */
} or_physics;

/* ---------------------------------------------------------------- 2D MLS-MPM (Flip) */
/* params: Flip.params words (f32 bits), at least 5: [dt, gx, gy, bulk, rho0, ...] (Flip.java:95-121). */
typedef struct {
    int nx, ny, np;
    float *x, *y, *u, *v, *m, *j, *c00, *c01, *c10, *c11;   /* SoA particles (caller-owned) */
    float *gm, *gmu, *gmv, *gu, *gv;                         /* grid, nx*ny (caller-owned) */
} or_flip2;

void or_flip2_clear(or_flip2* s);                                           /* Flip.java:226-235 */
void or_flip2_scatter(or_flip2* s, const float* params, or_physics ph);     /* Flip.java:269-303 */
void or_flip2_grid(or_flip2* s, const float* params, or_physics ph);        /* Flip.java:366-412 */
void or_flip2_advect(or_flip2* s, const float* params);                     /* Flip.java:494-559 */
void or_flip2_step(or_flip2* s, const float* params, or_physics ph);        /* FlipStep.step(): clear, scatter, grid, advect */
/* Flip.advectRelaxing (Flip.java:451-464, 512-543): J drawn toward rho0 / (the stencil's mass density) at the
 * params' RELAX word per second, where that density is at least OR_RELAX_MIN_DENSITY of rest; and FlipStep's
 * step built with relax. params: >= 12 words. */
#define OR_P_RELAX 11               /* Flip.java:113 */
#define OR_RELAX_MIN_DENSITY 0.8f   /* Flip.java:449 */
void or_flip2_advect_relaxing(or_flip2* s, const float* params);
void or_flip2_step_relaxing(or_flip2* s, const float* params, or_physics ph);

/* 2D sort key and stable counting sort (Scatter.java:458-502, FlipStep.java:183-192).
 * cells = (nx-1)(ny-1); starts has cells+1 words. The permutation is stable by key. */
int32_t or_cell2(float x, float y, int nx, int ny);                         /* Scatter.java:473-477 */
void or_sort2_keys(const float* x, const float* y, int64_t np, int nx, int ny, int32_t* keys);
/* counts -> starts (exclusive, length cells+1), then perm[dest] = src, stable. */
void or_counting_sort(const int32_t* keys, int64_t np, int64_t cells, int32_t* starts, int32_t* perm);
/* apply perm to nf float fields in place (tmp has np floats) */
void or_apply_perm(float** fields, int nf, const int32_t* perm, int64_t np, float* tmp);
void or_flip2_sort(or_flip2* s, int32_t* starts /* cells+1 */, int32_t* perm_scratch, float* tmp);

/* 2D bilinear P2G (Scatter.java:154-350): f32 in particle order, and the f64 answer
 * of ScatterTest.reference (ScatterTest.java:429-451). */
void or_scatter2_bilinear(int nx, int ny, const float* x, const float* y, const float* u, const float* v,
                          const float* m, int64_t np, float* gm, float* gmu, float* gmv);
void or_scatter2_bilinear_f64(int nx, int ny, const float* x, const float* y, const float* u, const float* v,
                              const float* m, int64_t np, double* gm, double* gmu, double* gmv);
/* Scatter.cellStarts (Scatter.java:484-502): returns -1 (and the offending index in *bad) if unsorted. */
int32_t or_cell_starts2(const float* x, const float* y, int64_t np, int nx, int ny, int32_t* starts, int64_t* bad);

/* Fixed-point bilinear P2G (FixedScatter.java:153-229), i32 wrapping registers. */
void or_fixed_scatter2(int nx, int ny, const float* x, const float* y, const float* u, const float* v,
                       const float* m, int64_t np, int mass_bits, int velocity_bits,
                       int32_t* gm, int32_t* gmu, int32_t* gmv);

/* ---------------------------------------------------------------- 3D MLS-MPM (Flip3) */
/* params: Flip3.params words: [dt, gx, gy, gz, bulk, rho0, sigma] (Flip3.java:55-64). */
typedef struct {
    int nx, ny, nz, np;
    float *x, *y, *z, *u, *v, *w, *m, *j;
    float *c[9];                                  /* c00 c01 c02 c10 c11 c12 c20 c21 c22 */
    float *gm, *gmu, *gmv, *gmw, *gu, *gv, *gw;   /* grid, nx*ny*nz */
} or_flip3;

void or_flip3_clear(or_flip3* s);                                            /* Flip3.java:163-172 */
void or_flip3_scatter(or_flip3* s, const float* params, or_physics ph);      /* Flip3.java:193-246 */
void or_fixed_scatter3(or_flip3* s, const float* params, or_physics ph, int64_t* q /* 4 * nodes */);
void or_flip3_grid(or_flip3* s, const float* params, or_physics ph);         /* Flip3.java:267-311 */
void or_flip3_advect(or_flip3* s, const float* params);                      /* Flip3.java:329-383, 644-655 */
void or_flip3_step(or_flip3* s, const float* params, or_physics ph);

/* Surface tension (particle/Tension3.java), the passes Flip3Step runs between the scatter and the grid when it
 * has tension (Flip3Step.java:88-109). Nodes (k*ny + j)*nx + i; every neighbour read held to [1, n-2]. */
#define OR_TENSION_BLURS 6          /* Flip.java:100 */
#define OR_MIN_COLOUR 0.3f          /* Tension.java:74 */
#define OR_MASS_FLOOR 0.3f          /* Tension.java:77 */
void or_tension3_blur(int nx, int ny, int nz, const float* src, float* dst, const float* params,
                      int scaled);                                           /* Tension3.java:73-107 */
/* The mass to a colour and OR_TENSION_BLURS blurs, ping-ponging c0 (first) and c1; returns the last written. */
const float* or_tension3_colour(int nx, int ny, int nz, const float* gm, const float* params, float* c0, float* c1);
void or_tension3_stress(int nx, int ny, int nz, const float* colour, float* stress /* 6 * nodes:
                        txx tyy tzz txy txz tyz */);                        /* Tension3.java:128-154 */
void or_tension3_force(int nx, int ny, int nz, const float* colour, const float* stress, const int at[3],
                       float force[3]);                                      /* Tension3.java:162-200 */
void or_flip3_grid_tension(or_flip3* s, const float* params, or_physics ph, const float* colour,
                           const float* stress);                             /* Flip3.java:258-310 */
/* Flip3Step with tension: clear, scatter, colour and blurs, stress, grid with tension, advect.
 * scratch: 8 * nodes floats. */
void or_flip3_step_tension(or_flip3* s, const float* params, or_physics ph, float* scratch);

/* The 3D sort key: the stencil base cell of Flip3.Stencil3 (Flip3.java:664-678), base
 * cells 0..n-3 per axis, linearised brick-major in 8x8x8 bricks (the reference has no
 * 3D sort; the key is defined here: bricks in x-fastest order, cells x-fastest within a brick, so each brick's
 * particles form one contiguous run). */
enum { OR_BRICK = 8, OR_BRICK_CELLS = 512 };
int32_t or_key3(float x, float y, float z, int nx, int ny, int nz);
int64_t or_key3_count(int nx, int ny, int nz);   /* number of keys (starts has this + 1 words) */
void or_flip3_sort(or_flip3* s, int32_t* starts, int32_t* keys, int32_t* perm, float* tmp);

/* ---------------------------------------------------------------- shallow water */
enum { OR_EDGE_WALL = 0, OR_EDGE_OPEN = 1 };
/* One dispatch of ShallowWater.kernel (ShallowWater.java:166-242) over all cells,
 * in cell order. edges: west, east, south, north. params: [g, courant, dx, dy, dry].
 * The atomics are restated as their sequential result. */
void or_swe_dispatch(int nx, int ny, const int32_t edges[4], const float* params,
                     const float* in_h, const float* in_hu, const float* in_hv,
                     float* out_h, float* out_hu, float* out_hv,
                     const int32_t* speed_in, int32_t* speed_out, int32_t* speed_clear,
                     const int32_t* budget_in, int32_t* budget_out, int32_t* clamped);
/* ShallowWater.fastestWave (ShallowWater.java:287-295): f32 bits. */
int32_t or_swe_fastest_wave(const float* h, const float* hu, const float* hv, int64_t n, double g, double dry);

/* ---------------------------------------------------------------- diagnostics */
typedef struct {
    double volume, min_depth, max_depth, max_speed, max_froude, max_courant;
    int32_t non_finite, negative, wet;
} or_swe_diag;
void or_swe_diagnostics(const float* h, const float* hu, const float* hv, int64_t n, double g, double dry,
                        double dt, double dx, double dy, or_swe_diag* out);          /* Diagnostics.java:43-81 */
typedef struct {
    double min_density, max_density, low_density, high_density, mach, courant;
    int32_t non_finite;
} or_particle_diag;
void or_particle_diagnostics(const float* j, int64_t n, double speed, double sound, double dt,
                             or_particle_diag* out);                                  /* ParticleDiagnostics.java:126-148 */

/* ---------------------------------------------------------------- CPU baseline (OpenMP) */
/* The same 3D / SWE step, threaded for timing on the host cores: P2G into per-thread
 * grids then a reduction; everything else a parallel loop. Returns threads used. */
int or_baseline_threads(void);
void or_flip3_step_omp(or_flip3* s, const float* params, or_physics ph, float* scratch_grids /* threads*4*nodes */);
/* The same with tension's passes (Flip3Step with tension); tension: 8 * nodes floats. */
void or_flip3_step_tension_omp(or_flip3* s, const float* params, or_physics ph, float* scratch_grids,
                               float* tension);
void or_swe_dispatch_omp(int nx, int ny, const int32_t edges[4], const float* params,
                         const float* in_h, const float* in_hu, const float* in_hv,
                         float* out_h, float* out_hu, float* out_hv,
                         const int32_t* speed_in, int32_t* speed_out, int32_t* speed_clear,
                         const int32_t* budget_in, int32_t* budget_out, int32_t* clamped);

#ifdef __cplusplus
}
#endif
#endif
