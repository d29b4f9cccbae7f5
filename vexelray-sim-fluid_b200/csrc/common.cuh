// common.cuh -- status handling, device helpers and shared constants of libvexfluid.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <string>

#include "../../include/vexfluid.h"

namespace vf {

// ------------------------------------------------------------------ errors
// The calling thread's last error message (vf_last_error copies it out).
void set_error(const char* fmt, ...);
const char* last_error();

#define VF_TRY_CUDA(expr)                                                                     \
    do {                                                                                      \
        cudaError_t e_ = (expr);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            ::vf::set_error("%s failed: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, \
                            __LINE__);                                                        \
            return VF_ECUDA;                                                                  \
        }                                                                                     \
    } while (0)

#define VF_CHECK_LAUNCH() VF_TRY_CUDA(cudaGetLastError())

#define VF_REQUIRE(cond, code, ...)       \
    do {                                  \
        if (!(cond)) {                    \
            ::vf::set_error(__VA_ARGS__); \
            return (code);                \
        }                                 \
    } while (0)

// Returns VF_ENODEV with a message when no sm_100 device is usable.
int32_t require_device();
// Number of SMs on the current device (148 on B200); cached.
int sm_count();

// cuTensorMapEncodeTiled from the driver (through the runtime's entry-point query, so the library needs no
// -lcuda); null when the driver does not offer it.
typedef CUresult (*EncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled tensor_map_encoder();

// Sets n floats at p to v on stream s (a kernel: no host buffer, no pageable copy).
cudaError_t fill_f32(float* p, int64_t n, float v, cudaStream_t s);

// Device status word bits, set by kernels' own bounds checks (never a trap).
enum : uint32_t {
    ST_OOB = 1u << 0,        // an index fell outside its buffer; the access was skipped
    ST_TIMEOUT = 1u << 1,    // a bounded wait gave up
    ST_RANK = 1u << 2,       // a sort rank fell outside its cell's run
    ST_POOL = 1u << 3        // a step needed more grid bricks than the sparse pool holds; their nodes were skipped
};

// ------------------------------------------------------------------ device helpers
__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

// One 16-byte vector reduction into global memory (sm_90+): {m, mu, mv, mw} of one node in one op.
__device__ __forceinline__ void red_add_v4(float4* addr, float a, float b, float c, float d) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(addr), "f"(a), "f"(b), "f"(c), "f"(d)
                 : "memory");
}

__device__ __forceinline__ void set_status(uint32_t* status, uint32_t bit) {
    if (status) atomicOr(status, bit);
}

// Quadratic B-spline weights (Flip.Stencil.weights, Flip.java:584-590 / Flip3.java:682-688):
// 1/2(3/2 - f)^2, 3/4 - (f - 1)^2, 1/2(f - 1/2)^2, in the reference's operand order.
__device__ __forceinline__ void bspline_weights(float f, float w[3]) {
    float a = __fsub_rn(1.5f, f);
    float c = __fsub_rn(f, 1.0f);
    float e = __fsub_rn(f, 0.5f);
    w[0] = __fmul_rn(0.5f, __fmul_rn(a, a));
    w[1] = __fsub_rn(0.75f, __fmul_rn(c, c));
    w[2] = __fmul_rn(0.5f, __fmul_rn(e, e));
}

// The pressure's impulse factor s = 4*dt*V0*J*p (Flip.java:283-286, Flip3.java:216-218).
// REF: J*p = B(1 - J). TAIT: p = k((1/J)^7 - 1), J*p = k(J^-6 - J).
__device__ __forceinline__ float impulse_factor(float dt, float m, float rho0, float bulk, float j, bool tait) {
    float jp;
    if (tait) {
        float r = __fdiv_rn(1.0f, j);
        float r2 = __fmul_rn(r, r);
        float r6 = __fmul_rn(__fmul_rn(r2, r2), r2);
        jp = __fmul_rn(bulk, __fsub_rn(r6, j));
    } else {
        jp = __fmul_rn(bulk, __fsub_rn(1.0f, j));
    }
    return __fmul_rn(__fmul_rn(4.0f, __fmul_rn(dt, __fdiv_rn(m, rho0))), jp);
}

// ------------------------------------------------------------------ grid-wide barrier (cooperative launches)
struct GridBarrier {
    unsigned count, gen;
    unsigned limit;   // polls before a waiter gives up; 0 = BAR_SPINS
    unsigned pad;
};

constexpr int BAR_SPINS = 1 << 24;   // x ~64 ns of __nanosleep: about a second

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid-wide barrier of a cooperative launch (all CTAs co-resident). The last CTA to arrive resets the
// count and advances the generation; the others wait for the generation to change, at most `limit` polls
// (BAR_SPINS when it is 0), after which they set ST_TIMEOUT. Returns false, to the whole CTA, when this CTA
// gave up: the caller then returns, so no CTA runs a phase whose inputs another CTA may not have finished.
// (A CTA that passes the barrier knows every CTA arrived, whatever others did after arriving.)
__device__ __forceinline__ bool grid_barrier(GridBarrier* b, uint32_t* status) {
    __shared__ int bar_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned gen = ld_acquire(&b->gen);
        __threadfence();
        if (atomicAdd(&b->count, 1u) == gridDim.x - 1) {
            atomicExch(&b->count, 0u);
            __threadfence();
            atomicAdd(&b->gen, 1u);
        } else {
            const unsigned limit = *(volatile unsigned*)&b->limit;
            const unsigned cap = limit ? limit : (unsigned)BAR_SPINS;
            unsigned spins = 0;
            while (ld_acquire(&b->gen) == gen) {
                if (++spins > cap) {
                    set_status(status, ST_TIMEOUT);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        bar_ok = ok;
    }
    __syncthreads();
    return bar_ok != 0;
}

inline int div_up(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// Params words (int32 bits) to floats, with the reference's validation.
inline float bits_to_float(int32_t b) {
    float f;
    memcpy(&f, &b, 4);
    return f;
}

// A device buffer owned by a handle.
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    int32_t alloc(size_t n) {
        release();
        if (n == 0) n = 16;
        cudaError_t e = cudaMalloc(&ptr, n);
        if (e != cudaSuccess) {
            ptr = nullptr;
            set_error("cudaMalloc(%zu) failed: %s", n, cudaGetErrorString(e));
            return VF_ENOMEM;
        }
        bytes = n;
        return VF_OK;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    template <class T>
    T* as() const {
        return reinterpret_cast<T*>(ptr);
    }
    ~DeviceBuffer() { release(); }
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
};

}  // namespace vf
