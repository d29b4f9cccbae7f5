// profiler.cuh -- per-handle kernel accounting: a launch count always, and when switched on,
// a CUDA event pair around every launch on the handle's stream, summed per kernel name.
#pragma once

#include <map>
#include <string>
#include <vector>

#include "common.cuh"

namespace vf {

struct Profiler {
    struct Rec {
        const char* name;
        cudaEvent_t a, b;
    };
    bool on = false;
    int64_t launches = 0;
    std::vector<Rec> pool;
    size_t used = 0;
    Rec* open = nullptr;
    std::map<std::string, std::pair<double, int64_t>> totals;   // name -> (ms, launches)

    void begin(const char* name, cudaStream_t s);
    void end(cudaStream_t s);
    void collect();
    void reset();
    int32_t read(int32_t idx, char* name, size_t cap, double* ms, int64_t* count);
    ~Profiler();
};

// Launches a kernel on a handle's stream with its profiler around it.
#define VF_LAUNCH(prof, name, stream, kernel, grid, block, smem, ...) \
    do {                                                             \
        (prof).begin(name, stream);                                  \
        kernel<<<grid, block, smem, stream>>>(__VA_ARGS__);          \
        (prof).end(stream);                                          \
        VF_CHECK_LAUNCH();                                           \
    } while (0)

}  // namespace vf
