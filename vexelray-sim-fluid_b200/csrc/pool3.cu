// pool3.cu -- sparse node storage for the 3D step: the page table of 8^3-node bricks and its pool.
//
// The reference plans this (docs/sparse-fluid.md:19-62: bricks, a dense page table over the domain, one pool,
// mark -> allocate -> sort -> scatter/update/gather over the active bricks) and has not built it. Here the sort
// already orders the particles brick-major and the tiled kernels already work brick by brick, so only where a
// node lives changes: node_addr looks its brick up in the page.
#include "mpm3_kernels.cuh"

namespace vf {

// One thread per (non-empty cell brick, one of the 8 node bricks its window reaches): mark that node brick.
__global__ void __launch_bounds__(256) k_pool_mark3(Step3 s, int* mark) {
    const Dims3 dm = s.d;
    const int na = *s.n_active;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < na * 8; t += gridDim.x * blockDim.x) {
        const int b = s.active[t >> 3], o = t & 7;
        const int bx = b % dm.nbx + (o & 1), by = (b / dm.nbx) % dm.nby + ((o >> 1) & 1),
                  bz = b / (dm.nbx * dm.nby) + (o >> 2);
        // the window of cell brick b is nodes 8b .. 8b + 9 along each axis; its second node brick may lie past
        // the domain's last node
        if (bx < s.pnx && by < s.pny && bz < s.pnz) mark[(bz * s.pny + by) * s.pnx + bx] = 1;
    }
}

// One block of 1024 threads: the marked bricks take slots 0.. in brick order, the rest -1, and the marks are
// cleared for the next step. A brick past the pool's capacity keeps its slot number, which node_addr refuses.
__global__ void __launch_bounds__(1024) k_pool_page3(int* mark, int* page, int npages, int* n_used, int cap,
                                                     uint32_t* status) {
    __shared__ int smem[33];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int seg = (npages + 31) / 32;
    const int lo = warp * seg, hi = min(lo + seg, npages);
    int live = 0;
    for (int base = lo; base < hi; base += 32) {
        const int i = base + lane;
        live += i < hi && mark[i] != 0;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) live += __shfl_xor_sync(0xffffffffu, live, o);
    int total;
    int slot = block_exclusive(lane == 0 ? live : 0, smem, &total);
    slot = __shfl_sync(0xffffffffu, slot, 0);
    for (int base = lo; base < hi; base += 32) {
        const int i = base + lane;
        const bool m = i < hi && mark[i] != 0;
        const unsigned set = __ballot_sync(0xffffffffu, m);
        if (i < hi) {
            page[i] = m ? slot + __popc(set & ((1u << lane) - 1u)) : -1;
            mark[i] = 0;
        }
        slot += __popc(set);
    }
    if (threadIdx.x == 0) {
        *n_used = min(total, cap);
        if (total > cap) set_status(status, ST_POOL);
    }
}

// Zeroes the slots the last scatter into this pool used.
__global__ void __launch_bounds__(256) k_pool_clear3(float4* pool, const int* n_used) {
    const int64_t n = (int64_t)*n_used * POOL_NODES;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        pool[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

__global__ void __launch_bounds__(256) k_pool_unpack3(Step3 s, float4* dense) {
    const Dims3 dm = s.d;
    const int64_t nodes = (int64_t)dm.nx * dm.ny * dm.nz;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nodes) return;
    const int gx = (int)(i % dm.nx), gy = (int)((i / dm.nx) % dm.ny), gz = (int)(i / ((int64_t)dm.nx * dm.ny));
    const float4* node = node_addr(s, gx, gy, gz);
    dense[i] = node ? *node : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

}  // namespace vf
