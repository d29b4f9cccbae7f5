// pdiag.cu -- ParticleDiagnostics.of (vexelray-sim-fluid-core/.../particle/ParticleDiagnostics.java:126-148) over
// a device-resident J, on the device.
//
// A valid J is finite and above zero (Float.isFinite && > 0); such floats order as their bit patterns do, so the
// count, the extremes and the two percentile ranks (the 1st and 99th, Math.min(n-1, (int)(p*n))) come out exact:
//   pass 0   count, min and max bits of the valid values, and a histogram of bits 31..21
//   select   per rank, the digit holding it (a scan of the histogram); the rank left within that digit
//   pass 1   a histogram of bits 20..10 over the values whose bits 31..21 are that digit; select
//   pass 2   bits 9..0 the same way; the prefix is then the rank's value, bit for bit
// Five launches over n floats and two 2048-bin histograms, then one 32-byte readback, instead of copying J to the
// host and sorting it.
#include <algorithm>

#include "common.cuh"

namespace vf {

struct PDiagState {
    unsigned n, minb, maxb, pad;
    unsigned prefix[2];
    unsigned rank[2];
};

constexpr int PD_BINS = 2048;

__device__ __forceinline__ void pd_digit(int pass, int& lo, int& width) {
    lo = pass == 0 ? 21 : pass == 1 ? 10 : 0;
    width = pass == 2 ? 10 : 11;
}

__global__ void __launch_bounds__(256) k_pdiag_pass(const float* __restrict__ j, int64_t n, int pass,
                                                    PDiagState* st, unsigned* hist) {
    __shared__ unsigned sh[2][PD_BINS];
    __shared__ unsigned red_n, red_min, red_max;
    for (int i = threadIdx.x; i < 2 * PD_BINS; i += blockDim.x) (&sh[0][0])[i] = 0;
    if (threadIdx.x == 0) {
        red_n = 0;
        red_min = 0xffffffffu;
        red_max = 0;
    }
    __syncthreads();
    int lo, width;
    pd_digit(pass, lo, width);
    const int high = lo + width;   // bits above the digit: the prefix selected so far
    const unsigned mask = (1u << width) - 1u;
    const unsigned pre0 = pass ? st->prefix[0] : 0u, pre1 = pass ? st->prefix[1] : 0u;
    unsigned cnt = 0, mn = 0xffffffffu, mx = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const unsigned b = __float_as_uint(j[i]);
        if (b - 1u >= 0x7f7fffffu) continue;   // not in (0, +inf): zero, negative, infinite or NaN
        const unsigned digit = (b >> lo) & mask;
        if (pass == 0) {
            cnt++;
            mn = min(mn, b);
            mx = max(mx, b);
            atomicAdd(&sh[0][digit], 1u);
        } else {
            const unsigned top = b >> high;
            if (top == pre0) atomicAdd(&sh[0][digit], 1u);
            if (top == pre1) atomicAdd(&sh[1][digit], 1u);
        }
    }
    if (pass == 0) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
            mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
            mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&red_n, cnt);
            atomicMin(&red_min, mn);
            atomicMax(&red_max, mx);
        }
    }
    __syncthreads();
    const int tables = pass == 0 ? 1 : 2;
    for (int i = threadIdx.x; i < tables * PD_BINS; i += blockDim.x) {
        const unsigned v = (&sh[0][0])[i];
        if (v) atomicAdd(&hist[i], v);
    }
    if (pass == 0 && threadIdx.x == 0 && red_n) {
        atomicAdd(&st->n, red_n);
        atomicMin(&st->minb, red_min);
        atomicMax(&st->maxb, red_max);
    }
}

// One CTA of PD_BINS / 2 threads (two bins each): for each rank, the digit whose cumulative count covers it.
constexpr int PD_SELECT = PD_BINS / 2;

__global__ void __launch_bounds__(PD_SELECT) k_pdiag_select(PDiagState* st, unsigned* hist, int pass) {
    __shared__ unsigned scan[PD_SELECT];
    __shared__ unsigned rank[2];
    const int t = threadIdx.x;
    if (pass == 0 && t == 0) {
        const unsigned n = st->n;
        // ParticleDiagnostics.percentile: Math.min(n - 1, (int) (p * n)); the 99th and the 1st
        const unsigned k99 = (unsigned)(0.99 * (double)n), k01 = (unsigned)(0.01 * (double)n);
        st->rank[0] = n ? min(n - 1, k99) : 0;
        st->rank[1] = n ? min(n - 1, k01) : 0;
    }
    __syncthreads();
    int lo, width;
    pd_digit(pass, lo, width);
    for (int q = 0; q < 2; q++) {
        const unsigned* hq = hist + (pass == 0 ? 0 : q * PD_BINS);
        const unsigned c0 = hq[2 * t], c1 = hq[2 * t + 1];
        scan[t] = c0 + c1;
        if (t == 0) rank[q] = st->rank[q];
        __syncthreads();
        for (int o = 1; o < PD_SELECT; o <<= 1) {   // inclusive scan of the pairs
            const unsigned v = t >= o ? scan[t - o] : 0u;
            __syncthreads();
            scan[t] += v;
            __syncthreads();
        }
        const unsigned below0 = scan[t] - c0 - c1, below1 = below0 + c0, r = rank[q];
        int hit = -1;
        unsigned below = 0;
        if (c0 && r >= below0 && r < below0 + c0) {
            hit = 2 * t;
            below = below0;
        } else if (c1 && r >= below1 && r < below1 + c1) {
            hit = 2 * t + 1;
            below = below1;
        }
        if (hit >= 0) {
            st->rank[q] = r - below;
            st->prefix[q] = pass == 0 ? (unsigned)hit : (st->prefix[q] << width) | (unsigned)hit;
        }
        __syncthreads();
    }
    for (int i = t; i < 2 * PD_BINS; i += PD_SELECT) hist[i] = 0;
}

// Scratch: PDiagState then 2 x PD_BINS unsigned.
size_t pdiag_scratch_bytes() { return sizeof(PDiagState) + 2 * PD_BINS * sizeof(unsigned); }

// The counts and the three order statistics of j's valid values, into host words:
// out = {n, min bits, max bits, bits at the 99th percentile rank, bits at the 1st}.
int32_t pdiag_run(const float* j, int64_t n, void* scratch, cudaStream_t s, unsigned out[5]) {
    PDiagState* st = reinterpret_cast<PDiagState*>(scratch);
    unsigned* hist = reinterpret_cast<unsigned*>(st + 1);
    const PDiagState init = {0u, 0xffffffffu, 0u, 0u, {0u, 0u}, {0u, 0u}};
    VF_TRY_CUDA(cudaMemcpyAsync(st, &init, sizeof init, cudaMemcpyHostToDevice, s));
    VF_TRY_CUDA(cudaMemsetAsync(hist, 0, 2 * PD_BINS * sizeof(unsigned), s));
    const int blocks = std::max(1, std::min(div_up(n, 256), sm_count() * 4));
    for (int pass = 0; pass < 3; pass++) {
        k_pdiag_pass<<<blocks, 256, 0, s>>>(j, n, pass, st, hist);
        k_pdiag_select<<<1, PD_SELECT, 0, s>>>(st, hist, pass);
    }
    VF_CHECK_LAUNCH();
    PDiagState got;
    VF_TRY_CUDA(cudaMemcpyAsync(&got, st, sizeof got, cudaMemcpyDeviceToHost, s));
    VF_TRY_CUDA(cudaStreamSynchronize(s));
    out[0] = got.n;
    out[1] = got.minb;
    out[2] = got.maxb;
    out[3] = got.prefix[0];
    out[4] = got.prefix[1];
    return VF_OK;
}

}  // namespace vf
