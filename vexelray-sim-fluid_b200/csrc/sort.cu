// sort.cu -- kernels of the stable counting sort by cell (see sort.cuh).
#include "sort.cuh"

namespace vf {

// ------------------------------------------------------------------ scans

__global__ void __launch_bounds__(1024) k_scan_single(int* __restrict__ counts, int* __restrict__ starts,
                                                      int64_t n) {
    __shared__ int smem[33];
    const int64_t per = (n + blockDim.x - 1) / blockDim.x;
    const int64_t lo = threadIdx.x * per;
    const int64_t hi = lo + per < n ? lo + per : n;
    int sum = 0;
    for (int64_t i = lo; i < hi; i++) sum += counts[i];
    int total;
    int run = block_exclusive(sum, smem, &total);
    for (int64_t i = lo; i < hi; i++) {
        int c = counts[i];
        starts[i] = run;
        run += c;
        counts[i] = 0;
    }
    if (threadIdx.x == 0) starts[n] = total;
}

// One block of 32 warps; warp w owns the contiguous segment [w*seg, (w+1)*seg) of the bricks and walks
// it 32 bricks at a time, so every load and store of a warp is one coalesced 128-byte line. Pass 1 sums
// each segment; a block scan gives each warp its offsets; pass 2 scans each 32-brick chunk with
// shuffles, writes the starts, appends the non-empty bricks in order and zeroes the counts.
__global__ void __launch_bounds__(1024) k_brick_scan(int* __restrict__ brick_count, int* __restrict__ brick_start,
                                                     int* __restrict__ active, int* __restrict__ n_active, int nb) {
    __shared__ int smem[33];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int seg = (nb + 31) / 32;
    const int lo = warp * seg, hi = min(lo + seg, nb);
    int sum = 0, live = 0;
    for (int base = lo; base < hi; base += 32) {
        const int i = base + lane;
        const int c = i < hi ? brick_count[i] : 0;
        sum += c;
        live += c > 0;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_xor_sync(0xffffffffu, sum, o);
        live += __shfl_xor_sync(0xffffffffu, live, o);
    }
    // one value per warp into the block scan (lane 0 carries it, the rest add nothing)
    int total, total_live;
    int run = block_exclusive(lane == 0 ? sum : 0, smem, &total);
    int slot = block_exclusive(lane == 0 ? live : 0, smem, &total_live);
    run = __shfl_sync(0xffffffffu, run, 0);
    slot = __shfl_sync(0xffffffffu, slot, 0);
    for (int base = lo; base < hi; base += 32) {
        const int i = base + lane;
        const int c = i < hi ? brick_count[i] : 0;
        const int inc = warp_inclusive(c);
        const unsigned nz = __ballot_sync(0xffffffffu, c > 0);
        if (i < hi) {
            brick_start[i] = run + inc - c;
            if (c > 0) active[slot + __popc(nz & ((1u << lane) - 1u))] = i;
            brick_count[i] = 0;
        }
        run += __shfl_sync(0xffffffffu, inc, 31);
        slot += __popc(nz);
    }
    if (threadIdx.x == 0) {
        brick_start[nb] = total;
        n_active[0] = total_live;
        n_active[2] = 0;   // the tiled gather's item counter for this list
    }
}

__global__ void __launch_bounds__(512) k_cell_scan(int* __restrict__ cell_count, int* __restrict__ cell_start,
                                                   int* __restrict__ cursor, const int* __restrict__ brick_start,
                                                   const int* __restrict__ active,
                                                   const int* __restrict__ n_active) {
    __shared__ int smem[33];
    const int na = *n_active;
    for (int a = blockIdx.x; a < na; a += gridDim.x) {
        const int b = active[a];
        const int64_t key = (int64_t)b * 512 + threadIdx.x;
        int c = cell_count[key];
        int total;
        int ex = block_exclusive(c, smem, &total);
        cell_start[key] = brick_start[b] + ex;
        if (cursor) cursor[key] = brick_start[b] + ex;
        cell_count[key] = 0;
    }
}

__global__ void k_permute(const int* __restrict__ key, const int* __restrict__ rank, const int* __restrict__ starts,
                          int* __restrict__ perm, int n, int64_t cells, uint32_t* status) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int k = key[i];
    if (k < 0 || (int64_t)k >= cells) {
        set_status(status, ST_OOB);
        return;
    }
    int d = starts[k] + rank[i];
    if (d < 0 || d >= n) {
        set_status(status, ST_RANK);
        return;
    }
    perm[d] = i;
}

__global__ void __launch_bounds__(256) k_permute_cursor(const int* __restrict__ key, int* __restrict__ cursor,
                                                       int* __restrict__ perm, int n, int64_t nkeys, uint32_t* status) {
    // PERMUTE_PER slots a thread, PERMUTE_PER x 256 a block; a warp's slots for one u are consecutive, so in the
    // last step's sorted order their keys come in runs: one cursor atomic per run, all of a thread's in flight
    // together before their ranks are read
    const unsigned all = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int base = blockIdx.x * (256 * PERMUTE_PER) + threadIdx.x;
    int k[PERMUTE_PER], leader[PERMUTE_PER], rank[PERMUTE_PER], got[PERMUTE_PER];
#pragma unroll
    for (int u = 0; u < PERMUTE_PER; u++) {
        const int i = base + u * 256;
        k[u] = i < n ? key[i] : -1;
        if (i < n && (k[u] < 0 || (int64_t)k[u] >= nkeys)) {
            set_status(status, ST_OOB);
            k[u] = -1;
        }
    }
#pragma unroll
    for (int u = 0; u < PERMUTE_PER; u++) {
        const int prev = __shfl_up_sync(all, k[u], 1);
        const unsigned starts = __ballot_sync(all, lane == 0 || prev != k[u]);
        leader[u] = 31 - __clz(starts & (0xffffffffu >> (31 - lane)));   // the run's first lane
        const unsigned above = starts & ~(0xffffffffu >> (31 - lane));    // run starts after this lane
        const int end = above ? __ffs(above) - 1 : 32;
        rank[u] = lane - leader[u];
        got[u] = (lane == leader[u] && k[u] >= 0) ? atomicAdd(&cursor[k[u]], end - leader[u]) : 0;
    }
#pragma unroll
    for (int u = 0; u < PERMUTE_PER; u++) {
        const int d = __shfl_sync(all, got[u], leader[u]) + rank[u];
        const int i = base + u * 256;
        if (k[u] < 0) continue;
        if (d < 0 || d >= n) {
            set_status(status, ST_RANK);
            continue;
        }
        perm[d] = i;
    }
}

// Insertion sort of a short run, ascending.
__device__ __forceinline__ void insertion_sort(int* a, int n) {
    for (int i = 1; i < n; i++) {
        int v = a[i];
        int j = i - 1;
        while (j >= 0 && a[j] > v) {
            a[j + 1] = a[j];
            j--;
        }
        a[j + 1] = v;
    }
}

__global__ void k_fixup_cells(int* __restrict__ perm, const int* __restrict__ starts, int64_t cells) {
    int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cells) return;
    int s0 = starts[c], s1 = starts[c + 1];
    if (s1 - s0 > 1) insertion_sort(perm + s0, s1 - s0);
}

// Runs up to this many particles per brick are fixed up in shared memory.
constexpr int FIXUP_CAP = 12288;

__global__ void __launch_bounds__(512) k_fixup_bricks(int* __restrict__ perm, const int* __restrict__ cell_start,
                                                      const int* __restrict__ brick_start,
                                                      const int* __restrict__ active,
                                                      const int* __restrict__ n_active) {
    extern __shared__ int run[];
    const int na = *n_active;
    for (int a = blockIdx.x; a < na; a += gridDim.x) {
        const int b = active[a];
        const int bs = brick_start[b], be = brick_start[b + 1];
        const int n = be - bs;
        const int64_t key = (int64_t)b * 512 + threadIdx.x;
        int s0 = cell_start[key];
        int s1 = threadIdx.x < 511 ? cell_start[key + 1] : be;
        s0 = max(s0, bs);   // a run always lies inside its brick's; clip anything else
        s1 = min(max(s1, s0), be);
        if (n <= FIXUP_CAP) {
            for (int i = threadIdx.x; i < n; i += blockDim.x) run[i] = perm[bs + i];
            __syncthreads();
            if (s1 - s0 > 1) insertion_sort(run + (s0 - bs), s1 - s0);
            __syncthreads();
            for (int i = threadIdx.x; i < n; i += blockDim.x) perm[bs + i] = run[i];
            __syncthreads();
        } else {
            if (s1 - s0 > 1) insertion_sort(perm + s0, s1 - s0);
        }
    }
}

__global__ void k_dense_starts3(const int* __restrict__ cell_start, const int* __restrict__ brick_start,
                                int* __restrict__ out, int64_t nkeys, int np) {
    int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k > nkeys) return;
    if (k == nkeys) {
        out[k] = np;
        return;
    }
    int64_t b = k >> 9;
    bool live = brick_start[b + 1] > brick_start[b];
    out[k] = live ? cell_start[k] : brick_start[b];
}

__global__ void k_gather_fields(const float* __restrict__ in, float* __restrict__ out, const int* __restrict__ perm,
                                int n, int64_t stride, int nf) {
    int d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= n) return;
    int s = perm[d];
    for (int f = 0; f < nf; f++) out[f * stride + d] = in[f * stride + s];
}

}  // namespace vf

