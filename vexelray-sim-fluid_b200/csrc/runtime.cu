// runtime.cu -- the library's plumbing: per-thread error messages, device checks, CUDA events
// for callers that time the handles' streams, and the per-handle kernel profiler.
#include <stdarg.h>

#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "profiler.cuh"

namespace vf {

// ------------------------------------------------------------------ errors and device

static thread_local char g_error[1024] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_error, sizeof g_error, fmt, ap);
    va_end(ap);
}

const char* last_error() { return g_error; }

int32_t require_device() {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        set_error("no CUDA device: %s", e == cudaSuccess ? "none found" : cudaGetErrorString(e));
        cudaGetLastError();
        return VF_ENODEV;
    }
    int dev = 0, major = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (major != 10) {
        set_error("libvexfluid is built for sm_100a (B200); device %d is compute capability %d.x", dev, major);
        return VF_ENODEV;
    }
    return VF_OK;
}

int sm_count() {
    static int cached = 0;
    if (!cached) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&cached, cudaDevAttrMultiProcessorCount, dev);
        if (cached <= 0) cached = 148;
    }
    return cached;
}

__global__ void k_fill_f32(float* p, int64_t n, float v) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = v;
}

cudaError_t fill_f32(float* p, int64_t n, float v, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    const int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)sm_count() * 8);
    k_fill_f32<<<blocks, 256, 0, s>>>(p, n, v);
    return cudaGetLastError();
}

EncodeTiled tensor_map_encoder() {
    static EncodeTiled fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiled)p;
        cudaGetLastError();
    }
    return fn;
}

// ------------------------------------------------------------------ profiler

Profiler::~Profiler() {
    for (auto& r : pool) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
}

void Profiler::begin(const char* name, cudaStream_t s) {
    launches++;
    if (!on) return;
    if (used == pool.size()) {
        Rec r{};
        cudaEventCreate(&r.a);
        cudaEventCreate(&r.b);
        pool.push_back(r);
    }
    Rec& r = pool[used++];
    r.name = name;
    cudaEventRecord(r.a, s);
    open = &r;
}

void Profiler::end(cudaStream_t s) {
    if (!on || !open) return;
    cudaEventRecord(open->b, s);
    open = nullptr;
}

void Profiler::collect() {
    if (used == 0) return;
    cudaEventSynchronize(pool[used - 1].b);
    for (size_t k = 0; k < used; k++) {
        float ms = 0;
        cudaEventElapsedTime(&ms, pool[k].a, pool[k].b);
        auto& t = totals[pool[k].name];
        t.first += ms;
        t.second += 1;
    }
    used = 0;
}

void Profiler::reset() {
    collect();
    totals.clear();
}

int32_t Profiler::read(int32_t idx, char* name, size_t cap, double* ms, int64_t* count) {
    collect();
    if (idx < 0 || idx >= (int32_t)totals.size()) {
        set_error("no profiled kernel %d", idx);
        return VF_EINVAL;
    }
    auto it = totals.begin();
    std::advance(it, idx);
    if (name && cap) {
        size_t n = std::min(cap - 1, it->first.size());
        memcpy(name, it->first.data(), n);
        name[n] = 0;
    }
    if (ms) *ms = it->second.first;
    if (count) *count = it->second.second;
    return VF_OK;
}

}  // namespace vf

// ------------------------------------------------------------------ C-ABI: errors and device

extern "C" int32_t vf_last_error(char* buf, size_t cap) {
    const char* e = vf::last_error();
    size_t n = strlen(e);
    if (buf && cap) {
        size_t k = n < cap - 1 ? n : cap - 1;
        memcpy(buf, e, k);
        buf[k] = 0;
    }
    return (int32_t)n;
}

extern "C" int32_t vf_version(void) { return 1; }

extern "C" int32_t vf_device_ok(void) { return vf::require_device() == VF_OK ? 1 : 0; }

extern "C" int32_t vf_binary_version(int32_t* out) {
    VF_REQUIRE(out, VF_EINVAL, "null argument");
    int32_t rc = vf::require_device();
    if (rc) return rc;
    cudaFuncAttributes attr{};
    VF_TRY_CUDA(cudaFuncGetAttributes(&attr, vf::k_fill_f32));
    *out = attr.binaryVersion;
    return VF_OK;
}

extern "C" int32_t vf_set_device(int32_t device) {
    VF_TRY_CUDA(cudaSetDevice(device));
    return vf::require_device();
}

extern "C" int32_t vf_event_create(void** ev) {
    VF_REQUIRE(ev, VF_EINVAL, "null argument");
    cudaEvent_t e;
    VF_TRY_CUDA(cudaEventCreate(&e));
    *ev = (void*)e;
    return VF_OK;
}

extern "C" int32_t vf_event_record(void* ev, void* stream) {
    VF_REQUIRE(ev, VF_EINVAL, "null event");
    VF_TRY_CUDA(cudaEventRecord((cudaEvent_t)ev, (cudaStream_t)stream));
    return VF_OK;
}

extern "C" int32_t vf_event_elapsed_ms(void* start, void* stop, float* ms) {
    VF_REQUIRE(start && stop && ms, VF_EINVAL, "null argument");
    VF_TRY_CUDA(cudaEventSynchronize((cudaEvent_t)stop));
    VF_TRY_CUDA(cudaEventElapsedTime(ms, (cudaEvent_t)start, (cudaEvent_t)stop));
    return VF_OK;
}

extern "C" void vf_event_destroy(void* ev) {
    if (ev) cudaEventDestroy((cudaEvent_t)ev);
}

extern "C" int32_t vf_host_register(void* ptr, size_t bytes) {
    VF_REQUIRE(ptr && bytes, VF_EINVAL, "null or empty range");
    VF_TRY_CUDA(cudaHostRegister(ptr, bytes, cudaHostRegisterDefault));
    return VF_OK;
}

extern "C" int32_t vf_host_unregister(void* ptr) {
    VF_REQUIRE(ptr, VF_EINVAL, "null pointer");
    VF_TRY_CUDA(cudaHostUnregister(ptr));
    return VF_OK;
}
