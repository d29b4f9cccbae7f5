// noalloc.cu -- vf_sort2_noalloc: the 2D stable sort by cell (the same result as vf_sort2) with every
// device buffer it needs taken from one fixed, file-scope device array instead of cudaMalloc.
//
// Who needs it: a caller that must not allocate device memory while it runs. Examples are a host
// that budgets all device memory up front (a game or a JVM application sharing the GPU with a
// renderer), and a real-time loop where cudaMalloc/cudaFree would synchronise the device and stall
// the frame. vf_sort2 allocates and frees its scratch on every call; this entry point does not.
//
// Limits and sharing:
//  * at most VF_SORT2_NOALLOC_MAX_PARTICLES particles and VF_SORT2_NOALLOC_MAX_CELLS cells,
//    (nx-1)*(ny-1); larger inputs are refused with VF_EINVAL before any device work;
//  * the array (about 7 MB) is part of the library image: every GPU that loads the library holds
//    it until the process exits;
//  * every call uses the same array and leaves its contents behind; the counts are cleared at the
//    start of each call. Calls that overlap on the GPU (from several host threads, or several
//    streams) race on the array and must be serialised by the caller;
//  * each call looks up the array's device address on the current device (cudaGetSymbolAddress, a
//    host-side lookup); the first call on a device also loads the library's module there, so make
//    that first call before any stream capture.

#include "sort.cuh"

using namespace vf;

namespace {

constexpr int64_t MAX_P = 1 << 18;       // particles
constexpr int64_t MAX_C = 1 << 18;       // cells
constexpr int64_t WORDS = 5 * MAX_P + 2 * MAX_C + 1 + 64;   // x y key rank perm | counts starts | status

// The scratch. In host code its name is only a host-side stand-in: kernels get the device address
// found by cudaGetSymbolAddress, never the symbol itself.
static __device__ __align__(256) int32_t g_sort2_scratch[WORDS];

// Scatter.cell (Scatter.java:473-477), counted with warp-aggregated atomics: the sort's first pass.
__global__ void __launch_bounds__(256) k_count_cells(const float* x, const float* y, int np, int nx, int ny,
                                                     int* counts, int* key, int* rank, int64_t cells,
                                                     uint32_t* status) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = i < np;
    int k = 0;
    if (valid) {
        float cx = clampf(x[i], 0.0f, (float)nx - 1.0f);
        float cy = clampf(y[i], 0.0f, (float)ny - 1.0f);
        k = (int)fminf(cy, (float)(ny - 2)) * (nx - 1) + (int)fminf(cx, (float)(nx - 2));
    }
    int r = warp_count(counts, k, valid, cells, status);
    if (valid) {
        key[i] = k;
        rank[i] = r;
    }
}

// The device address of the scratch on the current device. It is looked up on every call (a host-side table
// lookup, no allocation), so a module reloaded after cudaDeviceReset is found at its new address.
int32_t scratch_address(int32_t** out) {
    int dev = 0;
    VF_TRY_CUDA(cudaGetDevice(&dev));
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_sort2_scratch);
    if (e != cudaSuccess || !p) {
        set_error("cudaGetSymbolAddress of the sort scratch failed on device %d: %s", dev, cudaGetErrorString(e));
        return VF_ECUDA;
    }
    *out = (int32_t*)p;
    return VF_OK;
}

}  // namespace

extern "C" int32_t vf_sort2_noalloc(int32_t nx, int32_t ny, const float* x, const float* y, int64_t np,
                                    int32_t* perm, int32_t* starts) {
    VF_REQUIRE(x && y && perm && starts, VF_EINVAL, "null argument");
    VF_REQUIRE(nx >= 2 && ny >= 2, VF_EINVAL, "a grid needs at least two nodes each way, got %d x %d", nx, ny);
    VF_REQUIRE((int64_t)nx * ny <= INT32_MAX, VF_EINVAL,
               "a grid of %d x %d nodes has more than 2^31-1 nodes: its cell keys would not fit an int32", nx, ny);
    const int64_t cells = (int64_t)(nx - 1) * (ny - 1);
    VF_REQUIRE(np >= 1 && np <= MAX_P, VF_EINVAL,
               "vf_sort2_noalloc takes 1 to %lld particles, got %lld (its scratch is a fixed array; use vf_sort2)",
               (long long)MAX_P, (long long)np);
    VF_REQUIRE(cells <= MAX_C, VF_EINVAL,
               "vf_sort2_noalloc takes grids of at most %lld cells, got %lld (its scratch is a fixed array; use vf_sort2)",
               (long long)MAX_C, (long long)cells);
    int32_t rc = require_device();
    if (rc) return rc;
    int32_t* base = nullptr;
    if ((rc = scratch_address(&base))) return rc;
    float* dx = (float*)base;
    float* dy = (float*)(base + MAX_P);
    int* key = base + 2 * MAX_P;
    int* rank = base + 3 * MAX_P;
    int* dperm = base + 4 * MAX_P;
    int* counts = base + 5 * MAX_P;
    int* dstarts = counts + MAX_C;
    uint32_t* status = (uint32_t*)(dstarts + MAX_C + 1);
    const int n = (int)np;
    cudaStream_t s = 0;
    // the previous call's counts were zeroed by its scan, but a call that failed part-way may not have
    VF_TRY_CUDA(cudaMemsetAsync(counts, 0, (size_t)cells * 4, s));
    VF_TRY_CUDA(cudaMemsetAsync(status, 0, 4, s));
    VF_TRY_CUDA(cudaMemcpyAsync(dx, x, (size_t)n * 4, cudaMemcpyHostToDevice, s));
    VF_TRY_CUDA(cudaMemcpyAsync(dy, y, (size_t)n * 4, cudaMemcpyHostToDevice, s));
    k_count_cells<<<div_up(n, 256), 256, 0, s>>>(dx, dy, n, nx, ny, counts, key, rank, cells, status);
    k_scan_single<<<1, 1024, 0, s>>>(counts, dstarts, cells);
    k_permute<<<div_up(n, 256), 256, 0, s>>>(key, rank, dstarts, dperm, n, cells, status);
    k_fixup_cells<<<div_up(cells, 256), 256, 0, s>>>(dperm, dstarts, cells);
    VF_CHECK_LAUNCH();
    VF_TRY_CUDA(cudaMemcpyAsync(perm, dperm, (size_t)n * 4, cudaMemcpyDeviceToHost, s));
    VF_TRY_CUDA(cudaMemcpyAsync(starts, dstarts, (size_t)(cells + 1) * 4, cudaMemcpyDeviceToHost, s));
    uint32_t st = 0;
    VF_TRY_CUDA(cudaMemcpyAsync(&st, status, 4, cudaMemcpyDeviceToHost, s));
    VF_TRY_CUDA(cudaStreamSynchronize(s));
    VF_REQUIRE(st == 0, VF_EDEVICE, "a kernel flagged device status 0x%x", st);
    return VF_OK;
}
