// mpm2.cu -- the 2D particle step and the 2D scatter schedules, for sm_100a.
//   vf_mpm2_*        ParticleSimulation (vexelray-sim-fluid-gui/.../gui/ParticleSimulation.java) over
//                    FlipStep's passes (FlipStep.java:81-193): clear, scatter, grid, advect; the sort by
//                    cell every sort_every steps.
//   vf_scatter2      Scatter's four bilinear schedules (Scatter.java:154-350)
//   vf_fixed_scatter2  FixedScatter.kernel (FixedScatter.java:153-229)
//   vf_sort2         the sort by cell alone (SortTest.Sorter, SortTest.java:255-313)
// Reference paths: vexelray-sim-fluid-core/src/main/java/dev/vexelray/sim/fluid/particle/.
//
// Layout: particles are two sets (ping-pong) of 10 SoA f32 fields x y u v m j c00 c01 c10 c11
// (FlipStep.java:95-98); the grid is SoA gm gmu gmv gu gv over nx*ny nodes, row-major.
#include <vector>

#include "mpm2_device.cuh"
#include "sort.cuh"

using namespace vf;

namespace {

struct Grid2 {
    float *gm, *gmu, *gmv, *gu, *gv;
};

// Scatter.cell (Scatter.java:473-477): the bilinear cell, row-major over (nx-1)(ny-1).
__device__ __forceinline__ int cell2(float x, float y, int nx, int ny) {
    float cx = clampf(x, 0.0f, (float)nx - 1.0f);
    float cy = clampf(y, 0.0f, (float)ny - 1.0f);
    return (int)fminf(cy, (float)(ny - 2)) * (nx - 1) + (int)fminf(cx, (float)(nx - 2));
}

// ------------------------------------------------------------------ sort pass 1

__global__ void __launch_bounds__(256) k_key_count2(const float* x, const float* y, int np, int nx, int ny,
                                                    int* counts, int* key, int* rank, int64_t cells,
                                                    uint32_t* status) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = i < np;
    int k = valid ? cell2(x[i], y[i], nx, ny) : 0;
    int r = warp_count(counts, k, valid, cells, status);
    if (valid) {
        key[i] = k;
        rank[i] = r;
    }
}

// ------------------------------------------------------------------ the step

// Flip.scatter (Flip.java:269-303): mass, APIC momentum and the pressure's impulse on the 3x3
// stencil, segmented by the stencil's lower-left node.
__global__ void __launch_bounds__(256) k_flip2_scatter(const float* __restrict__ p, int64_t st, int np, int nx, int ny,
                                                       const Params2* __restrict__ prm, Grid2 g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float amt[27];
#pragma unroll
    for (int j = 0; j < 27; j++) amt[j] = 0.0f;
    int key = -1;
    if (i < np) {
        const Params2 q = *prm;
        Stencil2 s = stencil2(p[PX * st + i], p[PY * st + i], nx, ny);
        const float m = p[PM * st + i], u = p[PU * st + i], w = p[PV * st + i];
        const float c00 = p[PC00 * st + i], c01 = p[PC01 * st + i], c10 = p[PC10 * st + i], c11 = p[PC11 * st + i];
        const float sp = impulse_factor(q.dt, m, q.rho0, q.bulk, p[PJ * st + i], q.tait);
        key = s.base;
        scatter_amounts2(s, m, u, w, c00, c01, c10, c11, sp, amt);
    }
    if (segmented_sum<27>(amt, key) && key >= 0) {
#pragma unroll
        for (int k = 0; k < 9; k++) {
            const int node = key + (k / 3) * nx + k % 3;
            atomicAdd(&g.gm[node], amt[3 * k]);
            atomicAdd(&g.gmu[node], amt[3 * k + 1]);
            atomicAdd(&g.gmv[node], amt[3 * k + 2]);
        }
    }
}

// Flip.grid (Flip.java:366-412)
__global__ void __launch_bounds__(256) k_flip2_grid(int nx, int ny, const Params2* __restrict__ prm, Grid2 g) {
    const int node = blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= nx * ny) return;
    const float2 v = grid_velocity2(g.gm[node], g.gmu[node], g.gmv[node], node % nx, node / nx, nx, ny, *prm);
    g.gu[node] = v.x;
    g.gv[node] = v.y;
}

// Flip.advectBody (Flip.java:494-545)
__global__ void __launch_bounds__(256) k_flip2_advect(float* __restrict__ p, int64_t st, int np, int nx, int ny,
                                                      const Params2* __restrict__ prm, Grid2 g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const Params2 q = *prm;
    const float px = p[PX * st + i], py = p[PY * st + i];
    const Stencil2 s = stencil2(px, py, nx, ny);
    const Advected2 a = advect2(
        s, px, py, p[PJ * st + i], nx, ny, q,
        [&](int k) {
            const int node = s.base + (k / 3) * nx + k % 3;
            return make_float2(g.gu[node], g.gv[node]);
        },
        [&](int k) { return g.gm[s.base + (k / 3) * nx + k % 3]; });
    p[PX * st + i] = a.x;
    p[PY * st + i] = a.y;
    p[PU * st + i] = a.u;
    p[PV * st + i] = a.w;
    p[PC00 * st + i] = a.c00;
    p[PC01 * st + i] = a.c01;
    p[PC10 * st + i] = a.c10;
    p[PC11 * st + i] = a.c11;
    p[PJ * st + i] = a.j;
}

// ------------------------------------------------------------------ bilinear schedules (Scatter)

// Scatter.Particle.load (Scatter.java:547-556) and its deposit (559-596).
struct Bilinear {
    int col, row, corner;
    float fx, fy, m, u, v;
};

__device__ __forceinline__ Bilinear bilinear(const float* x, const float* y, const float* u, const float* v,
                                             const float* m, int p, int nx, int ny) {
    Bilinear b;
    float cx = clampf(x[p], 0.0f, (float)nx - 1.0f);
    float cy = clampf(y[p], 0.0f, (float)ny - 1.0f);
    b.col = (int)fminf(cx, (float)(nx - 2));
    b.row = (int)fminf(cy, (float)(ny - 2));
    b.fx = __fsub_rn(cx, (float)b.col);
    b.fy = __fsub_rn(cy, (float)b.row);
    b.m = m[p];
    b.u = u[p];
    b.v = v[p];
    b.corner = b.row * nx + b.col;
    return b;
}

__device__ __forceinline__ float corner_weight(const Bilinear& b, int k) {
    float wx = (k & 1) ? b.fx : __fsub_rn(1.0f, b.fx);
    float wy = (k >> 1) ? b.fy : __fsub_rn(1.0f, b.fy);
    return __fmul_rn(wx, wy);
}

// Scatter.kernel, Mode.GRID (Scatter.java:154-182)
__global__ void k_scatter2_grid(const float* x, const float* y, const float* u, const float* v, const float* m, int np,
                                int nx, int ny, float* gm, float* gmu, float* gmv) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    Bilinear b = bilinear(x, y, u, v, m, p, nx, ny);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float w = corner_weight(b, k);
        const float wm = __fmul_rn(w, b.m);
        const int node = b.corner + (k >> 1) * nx + (k & 1);
        atomicAdd(&gm[node], wm);
        atomicAdd(&gmu[node], __fmul_rn(wm, b.u));
        atomicAdd(&gmv[node], __fmul_rn(wm, b.v));
    }
}

// Scatter.preReduced (Scatter.java:199-254): a workgroup's deposits summed in a shared window of
// two rows of 257 nodes anchored at its first particle's cell; deposits outside it go straight
// to the grid; non-zero slots flushed with one atomic each.
constexpr int PR_WG = 256, PR_COLS = PR_WG + 1, PR_WINDOW = 2 * PR_COLS;

__global__ void __launch_bounds__(PR_WG) k_scatter2_prereduced(const float* x, const float* y, const float* u,
                                                              const float* v, const float* m, int np, int nx, int ny,
                                                              float* gm, float* gmu, float* gmv) {
    __shared__ float win[3][PR_WINDOW];
    const int lid = threadIdx.x;
    const int p = blockIdx.x * PR_WG + lid;
    const int anchor = blockIdx.x * PR_WG;
    Bilinear o = bilinear(x, y, u, v, m, anchor, nx, ny);
    for (int slot = lid; slot < PR_WINDOW; slot += PR_WG) win[0][slot] = win[1][slot] = win[2][slot] = 0.0f;
    __syncthreads();
    if (p < np) {
        Bilinear b = bilinear(x, y, u, v, m, p, nx, ny);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const float w = corner_weight(b, k);
            const float wm = __fmul_rn(w, b.m);
            const float a[3] = {wm, __fmul_rn(wm, b.u), __fmul_rn(wm, b.v)};
            const int dr = b.row + (k >> 1) - o.row;
            const int dc = b.col + (k & 1) - o.col;
            if (dr >= 0 && dr < 2 && dc >= 0 && dc < PR_COLS) {
                const int slot = dr * PR_COLS + dc;
                atomicAdd(&win[0][slot], a[0]);
                atomicAdd(&win[1][slot], a[1]);
                atomicAdd(&win[2][slot], a[2]);
            } else {
                const int node = b.corner + (k >> 1) * nx + (k & 1);
                atomicAdd(&gm[node], a[0]);
                atomicAdd(&gmu[node], a[1]);
                atomicAdd(&gmv[node], a[2]);
            }
        }
    }
    __syncthreads();
    for (int slot = lid; slot < PR_WINDOW; slot += PR_WG) {
        const int node = (o.row + slot / PR_COLS) * nx + (o.col + slot % PR_COLS);
        float* grids[3] = {gm, gmu, gmv};
        for (int f = 0; f < 3; f++) {
            const float sum = win[f][slot];
            if (sum != 0.0f) atomicAdd(&grids[f][node], sum);
        }
    }
}

// Scatter.gather (Scatter.java:267-310): one thread per node, over the particles of the up to four
// cells around it, sorted by cell with starts; no atomics, the same bits every run.
__global__ void k_scatter2_gather(const float* x, const float* y, const float* u, const float* v, const float* m,
                                  const int* starts, int nx, int ny, float* gm, float* gmu, float* gmv) {
    const int node = blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= nx * ny) return;
    const int cols = nx - 1;
    const int ni = node % nx, nj = node / nx;
    float sm = 0.0f, smu = 0.0f, smv = 0.0f;
    for (int dr = -1; dr <= 0; dr++) {
        for (int dc = -1; dc <= 0; dc++) {
            const bool east = dc == -1, north = dr == -1;
            const int cc = ni + dc, cr = nj + dr;
            if (cc < 0 || cc >= cols || cr < 0 || cr >= ny - 1) continue;
            const int cell = cr * cols + cc;
            for (int k = starts[cell]; k < starts[cell + 1]; k++) {
                const float px = clampf(x[k], 0.0f, (float)nx - 1.0f);
                const float py = clampf(y[k], 0.0f, (float)ny - 1.0f);
                const float fx = __fsub_rn(px, (float)cc), fy = __fsub_rn(py, (float)cr);
                const float w = __fmul_rn(east ? fx : __fsub_rn(1.0f, fx), north ? fy : __fsub_rn(1.0f, fy));
                const float wm = __fmul_rn(w, m[k]);
                sm = __fadd_rn(sm, wm);
                smu = __fadd_rn(smu, __fmul_rn(wm, u[k]));
                smv = __fadd_rn(smv, __fmul_rn(wm, v[k]));
            }
        }
    }
    gm[node] = sm;
    gmu[node] = smu;
    gmv[node] = smv;
}

// Scatter.segmented (Scatter.java:336-350): the run of a cell summed across the warp, then one
// atomic per node and field from the run's last lane.
__global__ void __launch_bounds__(256) k_scatter2_segmented(const float* x, const float* y, const float* u,
                                                            const float* v, const float* m, int np, int nx, int ny,
                                                            float* gm, float* gmu, float* gmv) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    float amt[12];
#pragma unroll
    for (int j = 0; j < 12; j++) amt[j] = 0.0f;
    int key = -1;
    if (p < np) {
        Bilinear b = bilinear(x, y, u, v, m, p, nx, ny);
        key = b.corner;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const float wm = __fmul_rn(corner_weight(b, k), b.m);
            amt[3 * k] = wm;
            amt[3 * k + 1] = __fmul_rn(wm, b.u);
            amt[3 * k + 2] = __fmul_rn(wm, b.v);
        }
    }
    if (segmented_sum<12>(amt, key) && key >= 0) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int node = key + (k >> 1) * nx + (k & 1);
            atomicAdd(&gm[node], amt[3 * k]);
            atomicAdd(&gmu[node], amt[3 * k + 1]);
            atomicAdd(&gmv[node], amt[3 * k + 2]);
        }
    }
}

// FixedScatter.kernel with Quanta (FixedScatter.java:153-229): integer shares, wrapping i32 adds.
__global__ void k_fixed_scatter2(const float* x, const float* y, const float* u, const float* v, const float* m,
                                 int np, int nx, int ny, float mscale, float vscale, int* gm, int* gmu, int* gmv) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    const int ONE = 1 << 10;
    Bilinear b = bilinear(x, y, u, v, m, p, nx, ny);
    const int mass = (int)__fmul_rn(b.m, mscale);
    const int uq = (int)__fmul_rn(b.u, vscale), vq = (int)__fmul_rn(b.v, vscale);
    const int ox = (int)__fmul_rn(b.fx, (float)ONE), oy = (int)__fmul_rn(b.fy, (float)ONE);
    const int high = mass / ONE, low = mass % ONE;
    int left = mass;
    int shares[4];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const int ax = (k & 1) ? ox : ONE - ox;
        const int ay = (k >> 1) ? oy : ONE - oy;
        const int q = ax * ay;
        const int share = (q * high + (q * low) / ONE) / ONE;
        left -= share;
        shares[k] = share;
    }
    shares[3] = left;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const int node = b.corner + (k >> 1) * nx + (k & 1);
        atomicAdd(&gm[node], shares[k]);
        atomicAdd(&gmu[node], (int)((unsigned)shares[k] * (unsigned)uq));
        atomicAdd(&gmv[node], (int)((unsigned)shares[k] * (unsigned)vq));
    }
}

// Upload helper.
template <class T>
int32_t upload(DeviceBuffer& b, const T* host, int64_t n, cudaStream_t s) {
    int32_t rc = b.alloc((size_t)n * sizeof(T));
    if (rc) return rc;
    VF_TRY_CUDA(cudaMemcpyAsync(b.ptr, host, (size_t)n * sizeof(T), cudaMemcpyHostToDevice, s));
    return VF_OK;
}

}  // namespace

// ------------------------------------------------------------------ the handle

struct vf_mpm2 {
    int nx, ny, np;
    uint32_t flags;
    int64_t cells, nodes, stride;
    cudaStream_t stream = nullptr;
    DeviceBuffer part[2];
    int cur = 0;
    DeviceBuffer key, rank, perm, counts, starts;
    DeviceBuffer grid;   // 5 * nodes floats: gm gmu gmv gu gv
    DeviceBuffer params, status;
    int64_t steps = 0;
    bool sorted = false;
    // vf_mpm2_set_graph: a sort and the sort_every steps after it, captured once per current particle set
    bool use_graph = false;
    cudaGraphExec_t block[2] = {nullptr, nullptr};
    int block_every = 0;   // the sort_every the blocks were captured for
};

namespace {

Grid2 grid_of(vf_mpm2* h) {
    float* g = h->grid.as<float>();
    return Grid2{g, g + h->nodes, g + 2 * h->nodes, g + 3 * h->nodes, g + 4 * h->nodes};
}

int32_t upload_params2(vf_mpm2* h, const int32_t* params, int32_t nparams) {
    VF_REQUIRE(params && nparams >= 5, VF_EINVAL, "Flip.params has at least 5 words, got %d", nparams);
    float w[5];
    for (int k = 0; k < 5; k++) w[k] = bits_to_float(params[k]);
    VF_REQUIRE(w[0] > 0 && w[3] >= 0 && w[4] > 0, VF_EINVAL,      // Flip.java:204-207
               "dt > 0, bulk >= 0 and rho0 > 0, got dt %g, bulk %g, rho0 %g", w[0], w[3], w[4]);
    Params2 p{w[0], w[1], w[2], w[3], w[4], (h->flags & VF_EOS_TAIT) ? 1 : 0,
              (int)((h->flags & VF_WALL_STICKY_MASK) >> VF_WALL_STICKY_SHIFT),
              nparams > 11 ? bits_to_float(params[11]) : 0.0f, (h->flags & VF_RELAX) ? 1 : 0};
    VF_TRY_CUDA(cudaMemcpyAsync(h->params.ptr, &p, sizeof p, cudaMemcpyHostToDevice, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return VF_OK;
}

// FlipStep.sort() (FlipStep.java:183-192): count, scan, permute, and the fields gathered into
// the other set, which becomes current (no copy back).
int32_t sort2(vf_mpm2* h) {
    float* in = h->part[h->cur].as<float>();
    float* out = h->part[h->cur ^ 1].as<float>();
    uint32_t* st = h->status.as<uint32_t>();
    k_key_count2<<<div_up(h->np, 256), 256, 0, h->stream>>>(in + PX * h->stride, in + PY * h->stride, h->np, h->nx,
                                                             h->ny, h->counts.as<int>(), h->key.as<int>(),
                                                             h->rank.as<int>(), h->cells, st);
    VF_CHECK_LAUNCH();
    k_scan_single<<<1, 1024, 0, h->stream>>>(h->counts.as<int>(), h->starts.as<int>(), h->cells);
    VF_CHECK_LAUNCH();
    k_permute<<<div_up(h->np, 256), 256, 0, h->stream>>>(h->key.as<int>(), h->rank.as<int>(), h->starts.as<int>(),
                                                          h->perm.as<int>(), h->np, h->cells, st);
    VF_CHECK_LAUNCH();
    k_fixup_cells<<<div_up(h->cells, 256), 256, 0, h->stream>>>(h->perm.as<int>(), h->starts.as<int>(), h->cells);
    VF_CHECK_LAUNCH();
    k_gather_fields<<<div_up(h->np, 256), 256, 0, h->stream>>>(in, out, h->perm.as<int>(), h->np, h->stride, NF2);
    VF_CHECK_LAUNCH();
    h->cur ^= 1;
    h->sorted = true;
    return VF_OK;
}

// FlipStep.step() (FlipStep.java:127-169)
int32_t step2(vf_mpm2* h) {
    float* p = h->part[h->cur].as<float>();
    Grid2 g = grid_of(h);
    const Params2* prm = h->params.as<Params2>();
    VF_TRY_CUDA(cudaMemsetAsync(g.gm, 0, (size_t)3 * h->nodes * 4, h->stream));
    k_flip2_scatter<<<div_up(h->np, 256), 256, 0, h->stream>>>(p, h->stride, h->np, h->nx, h->ny, prm, g);
    VF_CHECK_LAUNCH();
    k_flip2_grid<<<div_up(h->nodes, 256), 256, 0, h->stream>>>(h->nx, h->ny, prm, g);
    VF_CHECK_LAUNCH();
    k_flip2_advect<<<div_up(h->np, 256), 256, 0, h->stream>>>(p, h->stride, h->np, h->nx, h->ny, prm, g);
    VF_CHECK_LAUNCH();
    return VF_OK;
}

int32_t status2(vf_mpm2* h) {
    uint32_t st = 0;
    VF_TRY_CUDA(cudaMemcpyAsync(&st, h->status.ptr, 4, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    if (st) {
        VF_TRY_CUDA(cudaMemsetAsync(h->status.ptr, 0, 4, h->stream));
        set_error("a kernel flagged device status 0x%x", st);
        return VF_EDEVICE;
    }
    return VF_OK;
}

}  // namespace

extern "C" {

int32_t vf_mpm2_create(int32_t nx, int32_t ny, int32_t particles, uint32_t flags, vf_mpm2** out) {
    VF_REQUIRE(out, VF_EINVAL, "out is null");
    *out = nullptr;
    VF_REQUIRE(particles >= 1, VF_EINVAL, "a step needs particles, got %d", particles);
    VF_REQUIRE(nx >= 3 && ny >= 3, VF_EINVAL, "a grid needs at least three nodes each way, got %d x %d", nx, ny);
    VF_REQUIRE((int64_t)nx * ny <= INT32_MAX, VF_EINVAL,
               "a grid of %d x %d nodes has more than 2^31-1 nodes: its cell keys would not fit an int32", nx, ny);
    int32_t rc = require_device();
    if (rc) return rc;
    vf_mpm2* h = new vf_mpm2();
    h->nx = nx;
    h->ny = ny;
    h->np = particles;
    h->flags = flags;
    h->cells = (int64_t)(nx - 1) * (ny - 1);
    h->nodes = (int64_t)nx * ny;
    h->stride = ((int64_t)particles + 63) / 64 * 64;
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        set_error("cudaStreamCreate failed");
        return VF_ECUDA;
    }
    size_t pb = (size_t)h->stride * NF2 * 4;
    if ((rc = h->part[0].alloc(pb)) || (rc = h->part[1].alloc(pb)) || (rc = h->key.alloc((size_t)particles * 4)) ||
        (rc = h->rank.alloc((size_t)particles * 4)) || (rc = h->perm.alloc((size_t)particles * 4)) ||
        (rc = h->counts.alloc((size_t)h->cells * 4)) || (rc = h->starts.alloc((size_t)(h->cells + 1) * 4)) ||
        (rc = h->grid.alloc((size_t)5 * h->nodes * 4)) || (rc = h->params.alloc(sizeof(Params2))) ||
        (rc = h->status.alloc(16))) {
        vf_mpm2_destroy(h);
        return rc;
    }
    // ParticleSimulation's runner.clear(): the sort's counts must start at zero (ParticleSimulation.java:78)
    for (DeviceBuffer* b : {&h->part[0], &h->part[1], &h->counts, &h->starts, &h->grid, &h->status})
        cudaMemsetAsync(b->ptr, 0, b->bytes, h->stream);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
        vf_mpm2_destroy(h);
        set_error("clearing buffers failed");
        return VF_ECUDA;
    }
    *out = h;
    return VF_OK;
}

int32_t vf_mpm2_load(vf_mpm2* h, const float* x, const float* y, const float* u, const float* v, const float* m,
                     const int32_t* params, int32_t nparams) {
    VF_REQUIRE(h && x && y && u && v && m, VF_EINVAL, "null argument");
    int32_t rc = upload_params2(h, params, nparams);
    if (rc) return rc;
    float* base = h->part[h->cur].as<float>();
    const float* src[5] = {x, y, u, v, m};
    for (int f = 0; f < 5; f++)
        VF_TRY_CUDA(cudaMemcpyAsync(base + f * h->stride, src[f], (size_t)h->np * 4, cudaMemcpyHostToDevice, h->stream));
    VF_TRY_CUDA(fill_f32(base + PJ * h->stride, h->np, 1.0f, h->stream));
    VF_TRY_CUDA(cudaMemsetAsync(base + PC00 * h->stride, 0, (size_t)4 * h->stride * 4, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    h->steps = 0;
    return VF_OK;
}

int32_t vf_mpm2_params(vf_mpm2* h, const int32_t* params, int32_t nparams) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    return upload_params2(h, params, nparams);
}

}  // extern "C"

namespace {

// The block from a sort to the step before the next sort, captured for the current particle set (the sort moves
// the particles into the other set, so two blocks alternate); false if capture failed, with the state restored.
bool capture_block(vf_mpm2* h, int sort_every) {
    const int cur = h->cur;
    const bool sorted = h->sorted;
    if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    int32_t rc = sort2(h);
    for (int k = 0; !rc && k < sort_every; k++) rc = step2(h);
    cudaGraph_t graph = nullptr;
    const cudaError_t end = cudaStreamEndCapture(h->stream, &graph);
    cudaGraphExec_t exec = nullptr;
    const bool ok = !rc && end == cudaSuccess && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    h->cur = cur;
    h->sorted = sorted;
    if (!ok) return false;
    if (h->block[cur]) cudaGraphExecDestroy(h->block[cur]);
    h->block[cur] = exec;
    return true;
}

}  // namespace

extern "C" {

int32_t vf_mpm2_advance(vf_mpm2* h, int32_t count, int32_t sort_every) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    VF_REQUIRE(count >= 0 && sort_every >= 1, VF_EINVAL, "count >= 0 and sortEvery >= 1, got %d, %d", count,
               sort_every);
    for (int k = 0; k < count;) {
        int32_t rc;
        if (h->use_graph && h->steps % sort_every == 0 && count - k >= sort_every) {
            if (h->block_every != sort_every) {
                for (auto& b : h->block)
                    if (b) cudaGraphExecDestroy(b), b = nullptr;
                h->block_every = sort_every;
            }
            if (h->block[h->cur] || capture_block(h, sort_every)) {
                VF_TRY_CUDA(cudaGraphLaunch(h->block[h->cur], h->stream));
                h->cur ^= 1;
                h->sorted = true;
                h->steps += sort_every;
                k += sort_every;
                continue;
            }
            h->use_graph = false;   // this handle's steps do not capture; they run as launches
        }
        if (h->steps % sort_every == 0 && (rc = sort2(h))) return rc;
        if ((rc = step2(h))) return rc;
        h->steps++;
        k++;
    }
    return VF_OK;
}

int32_t vf_mpm2_set_graph(vf_mpm2* h, int32_t on) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    h->use_graph = on != 0;
    return VF_OK;
}

int32_t vf_mpm2_step(vf_mpm2* h) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    int32_t rc = step2(h);
    return rc ? rc : status2(h);
}

int32_t vf_mpm2_sort(vf_mpm2* h) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    int32_t rc = sort2(h);
    return rc ? rc : status2(h);
}

int32_t vf_mpm2_read(vf_mpm2* h, int32_t field, float* out, int64_t n) {
    VF_REQUIRE(h && out, VF_EINVAL, "null argument");
    const float* src;
    int64_t len;
    if (field >= VF2_X && field <= VF2_C11) {
        src = h->part[h->cur].as<float>() + (int64_t)field * h->stride;
        len = h->np;
    } else if (field >= VF2_GM && field <= VF2_GV) {
        src = h->grid.as<float>() + (int64_t)(field - VF2_GM) * h->nodes;
        len = h->nodes;
    } else {
        set_error("no field %d", field);
        return VF_EINVAL;
    }
    VF_REQUIRE(n == len, VF_EINVAL, "field %d holds %lld floats, got %lld", field, (long long)len, (long long)n);
    VF_TRY_CUDA(cudaMemcpyAsync(out, src, (size_t)len * 4, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return status2(h);
}

int32_t vf_mpm2_write(vf_mpm2* h, int32_t field, const float* in, int64_t n) {
    VF_REQUIRE(h && in, VF_EINVAL, "null argument");
    VF_REQUIRE(field >= VF2_X && field <= VF2_C11, VF_EINVAL, "no particle field %d", field);
    VF_REQUIRE(n == h->np, VF_EINVAL, "particle fields hold %d floats, got %lld", h->np, (long long)n);
    VF_TRY_CUDA(cudaMemcpyAsync(h->part[h->cur].as<float>() + (int64_t)field * h->stride, in, (size_t)n * 4,
                                cudaMemcpyHostToDevice, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return VF_OK;
}

int32_t vf_mpm2_read_starts(vf_mpm2* h, int32_t* out, int64_t n) {
    VF_REQUIRE(h && out, VF_EINVAL, "null argument");
    VF_REQUIRE(n == h->cells + 1, VF_EINVAL, "starts hold %lld words", (long long)(h->cells + 1));
    VF_REQUIRE(h->sorted, VF_ESTATE, "no sort has run");
    VF_TRY_CUDA(cudaMemcpyAsync(out, h->starts.ptr, (size_t)n * 4, cudaMemcpyDeviceToHost, h->stream));
    VF_TRY_CUDA(cudaStreamSynchronize(h->stream));
    return VF_OK;
}

int64_t vf_mpm2_steps(const vf_mpm2* h) { return h ? h->steps : 0; }

int32_t vf_mpm2_on_gpu(const vf_mpm2* h) { return h ? 1 : 0; }

void vf_mpm2_destroy(vf_mpm2* h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (auto& b : h->block)
        if (b) cudaGraphExecDestroy(b);
    for (DeviceBuffer* b : {&h->part[0], &h->part[1], &h->key, &h->rank, &h->perm, &h->counts, &h->starts, &h->grid,
                            &h->params, &h->status})
        b->release();
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

// ------------------------------------------------------------------ one-shot schedules

int32_t vf_scatter2(int32_t mode, int32_t nx, int32_t ny, const float* x, const float* y, const float* u,
                    const float* v, const float* m, int64_t np, float* gm, float* gmu, float* gmv) {
    VF_REQUIRE(x && y && u && v && m && gm && gmu && gmv, VF_EINVAL, "null argument");
    VF_REQUIRE(nx >= 2 && ny >= 2, VF_EINVAL, "a grid needs at least two nodes each way, got %d x %d", nx, ny);
    VF_REQUIRE((int64_t)nx * ny <= INT32_MAX, VF_EINVAL,
               "a grid of %d x %d nodes has more than 2^31-1 nodes: its cell keys would not fit an int32", nx, ny);
    VF_REQUIRE(mode >= VF_SCATTER_GRID && mode <= VF_SCATTER_SEGMENTED, VF_EINVAL, "no schedule %d", mode);
    VF_REQUIRE(np >= 0 && np < (1LL << 31), VF_EINVAL, "particle count %lld out of range", (long long)np);
    int32_t rc = require_device();
    if (rc) return rc;
    const int64_t nodes = (int64_t)nx * ny, cells = (int64_t)(nx - 1) * (ny - 1);
    cudaStream_t s = 0;
    DeviceBuffer dx, dy, du, dv, dm, grid, starts, keys;
    if ((rc = upload(dx, x, np, s)) || (rc = upload(dy, y, np, s)) || (rc = upload(du, u, np, s)) ||
        (rc = upload(dv, v, np, s)) || (rc = upload(dm, m, np, s)) || (rc = grid.alloc((size_t)3 * nodes * 4)))
        return rc;
    float* g = grid.as<float>();
    VF_TRY_CUDA(cudaMemsetAsync(g, 0, grid.bytes, s));
    const int n = (int)np;
    if (mode == VF_SCATTER_GATHER) {
        // Scatter.cellStarts refuses particles out of cell order (Scatter.java:484-502)
        std::vector<int> host((size_t)cells + 1, 0);
        int previous = 0;
        for (int64_t p = 0; p < np; p++) {
            float cx = fminf(fmaxf(x[p], 0.0f), (float)nx - 1.0f), cy = fminf(fmaxf(y[p], 0.0f), (float)ny - 1.0f);
            int c = (int)fminf(cy, (float)(ny - 2)) * (nx - 1) + (int)fminf(cx, (float)(nx - 2));
            VF_REQUIRE(c >= previous, VF_EINVAL,
                       "particle %lld is in cell %d after a particle in cell %d; the particles must be sorted by cell",
                       (long long)p, c, previous);
            previous = c;
            host[(size_t)c + 1]++;
        }
        for (int64_t c = 0; c < cells; c++) host[(size_t)c + 1] += host[(size_t)c];
        if ((rc = upload(starts, host.data(), cells + 1, s))) return rc;
        k_scatter2_gather<<<div_up(nodes, 256), 256, 0, s>>>(dx.as<float>(), dy.as<float>(), du.as<float>(),
                                                              dv.as<float>(), dm.as<float>(), starts.as<int>(), nx, ny,
                                                              g, g + nodes, g + 2 * nodes);
    } else if (n > 0) {
        if (mode == VF_SCATTER_GRID)
            k_scatter2_grid<<<div_up(n, 256), 256, 0, s>>>(dx.as<float>(), dy.as<float>(), du.as<float>(), dv.as<float>(),
                                                           dm.as<float>(), n, nx, ny, g, g + nodes, g + 2 * nodes);
        else if (mode == VF_SCATTER_PRE_REDUCED)
            k_scatter2_prereduced<<<div_up(n, PR_WG), PR_WG, 0, s>>>(dx.as<float>(), dy.as<float>(), du.as<float>(),
                                                                     dv.as<float>(), dm.as<float>(), n, nx, ny, g,
                                                                     g + nodes, g + 2 * nodes);
        else
            k_scatter2_segmented<<<div_up(n, 256), 256, 0, s>>>(dx.as<float>(), dy.as<float>(), du.as<float>(),
                                                                 dv.as<float>(), dm.as<float>(), n, nx, ny, g, g + nodes,
                                                                 g + 2 * nodes);
    }
    VF_CHECK_LAUNCH();
    VF_TRY_CUDA(cudaMemcpyAsync(gm, g, (size_t)nodes * 4, cudaMemcpyDeviceToHost, s));
    VF_TRY_CUDA(cudaMemcpyAsync(gmu, g + nodes, (size_t)nodes * 4, cudaMemcpyDeviceToHost, s));
    VF_TRY_CUDA(cudaMemcpyAsync(gmv, g + 2 * nodes, (size_t)nodes * 4, cudaMemcpyDeviceToHost, s));
    VF_TRY_CUDA(cudaStreamSynchronize(s));
    return VF_OK;
}

int32_t vf_fixed_scatter2(int32_t nx, int32_t ny, const float* x, const float* y, const float* u, const float* v,
                          const float* m, int64_t np, int32_t mass_bits, int32_t velocity_bits, int32_t* gm,
                          int32_t* gmu, int32_t* gmv) {
    VF_REQUIRE(x && y && u && v && m && gm && gmu && gmv, VF_EINVAL, "null argument");
    VF_REQUIRE(nx >= 2 && ny >= 2, VF_EINVAL, "a grid needs at least two nodes each way");
    VF_REQUIRE((int64_t)nx * ny <= INT32_MAX, VF_EINVAL,
               "a grid of %d x %d nodes has more than 2^31-1 nodes: its cell keys would not fit an int32", nx, ny);
    // FixedPoint (FixedScatter.java:96-101)
    VF_REQUIRE(mass_bits >= 0 && velocity_bits >= 0 && mass_bits <= 30 && velocity_bits <= 30, VF_EINVAL,
               "bits out of range: %d, %d", mass_bits, velocity_bits);
    int32_t rc = require_device();
    if (rc) return rc;
    const int64_t nodes = (int64_t)nx * ny;
    cudaStream_t s = 0;
    DeviceBuffer dx, dy, du, dv, dm, grid;
    if ((rc = upload(dx, x, np, s)) || (rc = upload(dy, y, np, s)) || (rc = upload(du, u, np, s)) ||
        (rc = upload(dv, v, np, s)) || (rc = upload(dm, m, np, s)) || (rc = grid.alloc((size_t)3 * nodes * 4)))
        return rc;
    int* g = grid.as<int>();
    VF_TRY_CUDA(cudaMemsetAsync(g, 0, grid.bytes, s));
    if (np > 0)
        k_fixed_scatter2<<<div_up(np, 256), 256, 0, s>>>(dx.as<float>(), dy.as<float>(), du.as<float>(), dv.as<float>(),
                                                         dm.as<float>(), (int)np, nx, ny, ldexpf(1.0f, mass_bits),
                                                         ldexpf(1.0f, velocity_bits), g, g + nodes, g + 2 * nodes);
    VF_CHECK_LAUNCH();
    VF_TRY_CUDA(cudaMemcpyAsync(gm, g, (size_t)nodes * 4, cudaMemcpyDeviceToHost, s));
    VF_TRY_CUDA(cudaMemcpyAsync(gmu, g + nodes, (size_t)nodes * 4, cudaMemcpyDeviceToHost, s));
    VF_TRY_CUDA(cudaMemcpyAsync(gmv, g + 2 * nodes, (size_t)nodes * 4, cudaMemcpyDeviceToHost, s));
    VF_TRY_CUDA(cudaStreamSynchronize(s));
    return VF_OK;
}

int32_t vf_sort2(int32_t nx, int32_t ny, const float* x, const float* y, int64_t np, int32_t* perm, int32_t* starts) {
    VF_REQUIRE(x && y && perm && starts, VF_EINVAL, "null argument");
    VF_REQUIRE(nx >= 2 && ny >= 2, VF_EINVAL, "a grid needs at least two nodes each way");
    VF_REQUIRE((int64_t)nx * ny <= INT32_MAX, VF_EINVAL,
               "a grid of %d x %d nodes has more than 2^31-1 nodes: its cell keys would not fit an int32", nx, ny);
    VF_REQUIRE(np >= 1 && np < (1LL << 31), VF_EINVAL, "particle count %lld out of range", (long long)np);
    int32_t rc = require_device();
    if (rc) return rc;
    const int64_t cells = (int64_t)(nx - 1) * (ny - 1);
    cudaStream_t s = 0;
    DeviceBuffer dx, dy, counts, dstarts, key, rank, dperm, status;
    if ((rc = upload(dx, x, np, s)) || (rc = upload(dy, y, np, s)) || (rc = counts.alloc((size_t)cells * 4)) ||
        (rc = dstarts.alloc((size_t)(cells + 1) * 4)) || (rc = key.alloc((size_t)np * 4)) ||
        (rc = rank.alloc((size_t)np * 4)) || (rc = dperm.alloc((size_t)np * 4)) || (rc = status.alloc(16)))
        return rc;
    VF_TRY_CUDA(cudaMemsetAsync(counts.ptr, 0, counts.bytes, s));
    VF_TRY_CUDA(cudaMemsetAsync(status.ptr, 0, status.bytes, s));
    const int n = (int)np;
    k_key_count2<<<div_up(n, 256), 256, 0, s>>>(dx.as<float>(), dy.as<float>(), n, nx, ny, counts.as<int>(),
                                                 key.as<int>(), rank.as<int>(), cells, status.as<uint32_t>());
    k_scan_single<<<1, 1024, 0, s>>>(counts.as<int>(), dstarts.as<int>(), cells);
    k_permute<<<div_up(n, 256), 256, 0, s>>>(key.as<int>(), rank.as<int>(), dstarts.as<int>(), dperm.as<int>(), n,
                                             cells, status.as<uint32_t>());
    k_fixup_cells<<<div_up(cells, 256), 256, 0, s>>>(dperm.as<int>(), dstarts.as<int>(), cells);
    VF_CHECK_LAUNCH();
    VF_TRY_CUDA(cudaMemcpyAsync(perm, dperm.ptr, (size_t)np * 4, cudaMemcpyDeviceToHost, s));
    VF_TRY_CUDA(cudaMemcpyAsync(starts, dstarts.ptr, (size_t)(cells + 1) * 4, cudaMemcpyDeviceToHost, s));
    uint32_t st = 0;
    VF_TRY_CUDA(cudaMemcpyAsync(&st, status.ptr, 4, cudaMemcpyDeviceToHost, s));
    VF_TRY_CUDA(cudaStreamSynchronize(s));
    VF_REQUIRE(st == 0, VF_EDEVICE, "a kernel flagged device status 0x%x", st);
    return VF_OK;
}

}  // extern "C"
