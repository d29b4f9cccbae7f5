// sort.cuh -- the counting sort by cell, shared by the 2D and 3D particle steps.
//
// The reference sorts with SupirVast's CountingSort (count -> 3 scan passes -> permute,
// FlipStep.java:183-192): counts[key]++ by atomics whose returned value is the rank, so the
// order within a cell is whatever order the atomics ran in (SortTest.java:121-134). Here the
// sort is defined as STABLE (ties keep their input order), and reproduced bit-exactly:
//
//   count    key per particle; counts[key] += 1 with warp-aggregated atomics (__match_any);
//            the returned rank is provisional
//   scan     counts -> exclusive starts (cells + 1 words, Scatter.cellStarts' layout);
//            counts are zeroed in the same pass, as the reference's last scan pass does
//   permute  perm[starts[key] + rank] = i
//   fix-up   each cell's run of perm sorted ascending, which makes the permutation stable
//
// The particles' fields are then gathered through perm by the next pass that reads them, so
// no separate copy-back pass exists (Flip.copy, Flip.java:632-640, is not needed).
#pragma once

#include "common.cuh"

namespace vf {

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// Adds one to counts[key] for every lane with valid set, one atomic per distinct key in the warp,
// and returns the lane's provisional rank (0 for invalid lanes). Must be called by all 32 lanes.
__device__ __forceinline__ int warp_count(int* counts, int key, bool valid, int64_t limit, uint32_t* status) {
    const unsigned all = 0xffffffffu;
    int k = valid ? key : -1;
    unsigned peers = __match_any_sync(all, k);
    int leader = __ffs(peers) - 1;
    int lane = lane_id();
    int below = __popc(peers & ((1u << lane) - 1u));
    int base = 0;
    if (lane == leader && k >= 0) {
        if ((int64_t)k < limit) base = atomicAdd(&counts[k], __popc(peers));
        else set_status(status, ST_OOB);
    }
    base = __shfl_sync(all, base, leader);
    return base + below;
}

// warp_count for keys that mostly come in runs (particles in slot order, sorted by the last step's keys): one
// atomic per run of equal consecutive keys instead of a match over the warp. A key that appears in two runs of the
// warp takes two atomics; the ranks are still distinct, and as provisional as warp_count's.
__device__ __forceinline__ int warp_count_runs(int* counts, int key, bool valid, int64_t limit, uint32_t* status) {
    const unsigned all = 0xffffffffu;
    const int lane = lane_id();
    const int k = valid ? key : -1;
    const int prev = __shfl_up_sync(all, k, 1);
    const unsigned starts = __ballot_sync(all, lane == 0 || prev != k);
    const int leader = 31 - __clz(starts & (0xffffffffu >> (31 - lane)));   // the run's first lane
    const unsigned above = starts & ~(0xffffffffu >> (31 - lane));          // run starts after this lane
    const int end = above ? __ffs(above) - 1 : 32;
    int base = 0;
    if (lane == leader && k >= 0) {
        if ((int64_t)k < limit) base = atomicAdd(&counts[k], end - leader);
        else set_status(status, ST_OOB);
    }
    base = __shfl_sync(all, base, leader);
    return base + (lane - leader);
}

// Adds one to counts[key] for every valid lane, aggregated per distinct key; no rank.
__device__ __forceinline__ void warp_tally(int* counts, int key, bool valid, int64_t limit, uint32_t* status) {
    const unsigned all = 0xffffffffu;
    int k = valid ? key : -1;
    unsigned peers = __match_any_sync(all, k);
    int leader = __ffs(peers) - 1;
    if (lane_id() == leader && k >= 0) {
        if ((int64_t)k < limit) atomicAdd(&counts[k], __popc(peers));
        else set_status(status, ST_OOB);
    }
}

// Inclusive scan of one int across a warp.
__device__ __forceinline__ int warp_inclusive(int v) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        int u = __shfl_up_sync(0xffffffffu, v, d);
        if (lane_id() >= d) v += u;
    }
    return v;
}

// Exclusive scan of one int across the block (blockDim.x a multiple of 32, <= 1024). Returns the
// exclusive prefix; *total gets the block's sum. Uses 33 ints of shared memory at smem.
__device__ __forceinline__ int block_exclusive(int v, int* smem, int* total) {
    int lane = lane_id(), warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int inc = warp_inclusive(v);
    if (lane == 31) smem[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        int s = lane < nw ? smem[lane] : 0;
        int si = warp_inclusive(s);
        if (lane < nw) smem[lane] = si - s;
        if (lane == 31) smem[32] = si;
    }
    __syncthreads();
    int r = smem[warp] + inc - v;
    *total = smem[32];
    __syncthreads();
    return r;
}

// counts[0..n) -> starts[0..n] exclusive (starts[n] = total), counts zeroed. One block of 1024
// threads; thread t owns the contiguous range [t*per, (t+1)*per).
__global__ void k_scan_single(int* __restrict__ counts, int* __restrict__ starts, int64_t n);

// The 3D brick level: brick_count[nb] -> brick_start[nb+1], the list of non-empty bricks in
// index order (active[0..*n_active)), brick_count zeroed, and n_active[2] (the tiled gather's item counter for
// this list) zeroed. One block of 1024 threads.
__global__ void k_brick_scan(int* __restrict__ brick_count, int* __restrict__ brick_start,
                             int* __restrict__ active, int* __restrict__ n_active, int nb);

// The 3D cell level, one block of 512 threads per non-empty brick: the brick's 512 cell counts
// -> cell_start (offset by brick_start) and, if given, a copy in cursor; counts zeroed.
__global__ void k_cell_scan(int* __restrict__ cell_count, int* __restrict__ cell_start, int* __restrict__ cursor,
                            const int* __restrict__ brick_start, const int* __restrict__ active,
                            const int* __restrict__ n_active);

// perm[cursor[key[i]]++] = i, the cursor bumped once per run of equal keys in a warp: the permutation with
// provisional (unstable) order within a cell, for counts that were tallied without ranks. PERMUTE_PER slots a
// thread, blocks of 256 threads: launch div_up(n, 256 * PERMUTE_PER) blocks.
constexpr int PERMUTE_PER = 4;
__global__ void k_permute_cursor(const int* __restrict__ key, int* __restrict__ cursor, int* __restrict__ perm, int n,
                                 int64_t nkeys, uint32_t* status);

// Insertion sort of a short run, ascending (the stable order's fix-up of one cell).
__device__ __forceinline__ void insertion_sort_run(int* a, int n) {
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

// perm[starts[key[i]] + rank[i]] = i.
__global__ void k_permute(const int* __restrict__ key, const int* __restrict__ rank,
                          const int* __restrict__ starts, int* __restrict__ perm, int n, int64_t cells,
                          uint32_t* status);

// Sorts each cell's run of perm ascending, one thread per cell (2D: cells small, runs short).
__global__ void k_fixup_cells(int* __restrict__ perm, const int* __restrict__ starts, int64_t cells);

// The same per brick (3D): the brick's run staged in shared memory, one thread per cell.
__global__ void k_fixup_bricks(int* __restrict__ perm, const int* __restrict__ cell_start,
                               const int* __restrict__ brick_start, const int* __restrict__ active,
                               const int* __restrict__ n_active);

// Dense cell starts of the 3D key space from the brick-level representation (for readback).
__global__ void k_dense_starts3(const int* __restrict__ cell_start, const int* __restrict__ brick_start,
                                int* __restrict__ out, int64_t nkeys, int np);

// out[f*stride + d] = in[f*stride + perm[d]] for nf fields.
__global__ void k_gather_fields(const float* __restrict__ in, float* __restrict__ out,
                                const int* __restrict__ perm, int n, int64_t stride, int nf);

}  // namespace vf
