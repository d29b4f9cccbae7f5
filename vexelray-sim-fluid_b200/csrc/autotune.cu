// autotune.cu -- the batched 2D step's tuner: per scene key, the P2G/G2P tile shape; per batch, the
// CTA size; both kept in a JSON cache so a later run on the same device skips the timing.
//
// Key of a scene: (particles per occupied stencil cell, rounded to a power of two; max(nx, ny), rounded up
// to a power of two). A tile shape is timed on a batch of up to 8 scenes of the key, whole steps (sort,
// scatter, gather: the tile shape changes all three), with CUDA events around graph replays after a
// warm-up. The CTA size is timed on up to 64 of the batch's scenes, drawn across its keys.
//
// Cache file: a JSON object {"format": ..., "entries": [...]}, one entry per line, written whole each time:
//   {"device": "<name>", "ppc": P, "n": N, "tile_x": X, "tile_y": Y, "us_per_step": T}
//   {"device": "<name>", "keys": "P/N P/N ...", "block": B, "us_per_step": T}
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "common.cuh"

using namespace vf;

namespace {

constexpr int TUNE_SCENES = 8;     // scenes per tile trial
constexpr int BLOCK_SCENES = 64;   // scenes per block trial
constexpr int WARM_STEPS = 3;
constexpr int TIMED_STEPS = 32;    // two graph replays

const int TILES[][2] = VF_BATCH_TILES;
const int BLOCKS[] = VF_BATCH_BLOCKS;

struct TileEntry {
    std::string device;
    int ppc, n, tx, ty;
    double us;
};

struct BlockEntry {
    std::string device;
    std::string keys;
    int block;
    double us;
};

struct Cache {
    std::vector<TileEntry> tiles;
    std::vector<BlockEntry> blocks;
};

bool field_str(const std::string& line, const char* name, std::string* out) {
    const std::string pat = std::string("\"") + name + "\": \"";
    size_t a = line.find(pat);
    if (a == std::string::npos) return false;
    a += pat.size();
    size_t b = line.find('"', a);
    if (b == std::string::npos) return false;
    *out = line.substr(a, b - a);
    return true;
}

bool field_num(const std::string& line, const char* name, double* out) {
    const std::string pat = std::string("\"") + name + "\": ";
    size_t a = line.find(pat);
    if (a == std::string::npos) return false;
    return sscanf(line.c_str() + a + pat.size(), "%lf", out) == 1;
}

Cache read_cache(const char* path) {
    Cache c;
    if (!path) return c;
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
        std::string dev, keys;
        double ppc, n, tx, ty, us, block;
        if (!field_str(line, "device", &dev)) continue;
        if (field_num(line, "ppc", &ppc) && field_num(line, "n", &n) && field_num(line, "tile_x", &tx) &&
            field_num(line, "tile_y", &ty) && field_num(line, "us_per_step", &us))
            c.tiles.push_back({dev, (int)ppc, (int)n, (int)tx, (int)ty, us});
        else if (field_str(line, "keys", &keys) && field_num(line, "block", &block) &&
                 field_num(line, "us_per_step", &us))
            c.blocks.push_back({dev, keys, (int)block, us});
    }
    return c;
}

int32_t write_cache(const char* path, const Cache& c) {
    if (!path) return VF_OK;
    std::ostringstream o;
    o << "{\"format\": \"vexfluid-batch2-autotune-1\", \"entries\": [\n";
    size_t k = 0, total = c.tiles.size() + c.blocks.size();
    char buf[512];
    for (const TileEntry& e : c.tiles) {
        snprintf(buf, sizeof buf,
                 "{\"device\": \"%s\", \"ppc\": %d, \"n\": %d, \"tile_x\": %d, \"tile_y\": %d, \"us_per_step\": %.3f}",
                 e.device.c_str(), e.ppc, e.n, e.tx, e.ty, e.us);
        o << buf << (++k < total ? ",\n" : "\n");
    }
    for (const BlockEntry& e : c.blocks) {
        o << "{\"device\": \"" << e.device << "\", \"keys\": \"" << e.keys << "\", \"block\": " << e.block;
        snprintf(buf, sizeof buf, ", \"us_per_step\": %.3f}", e.us);
        o << buf << (++k < total ? ",\n" : "\n");
    }
    o << "]}\n";
    std::ofstream f(path, std::ios::trunc);
    if (!f) {
        set_error("cannot write the autotune cache %s", path);
        return VF_EINVAL;
    }
    f << o.str();
    return f ? VF_OK : VF_EINVAL;
}

int pow2_round(double v) {   // the nearest power of two (in log), at least 1
    if (!(v > 1)) return 1;
    return 1 << (int)std::lround(std::log2(v));
}

int pow2_up(int v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

// Particles per occupied stencil cell of one scene (the cell stencil2 computes, Flip.java:572-581).
double scene_ppc(const vf_scene2& s, const float* x, const float* y) {
    const int cols = s.nx - 2, rows = s.ny - 2;
    std::vector<uint8_t> seen((size_t)cols * rows, 0);
    int64_t occupied = 0;
    for (int i = 0; i < s.particles; i++) {
        float px = std::min(std::max(x[i], 0.5f), (float)s.nx - 1.5f);
        float py = std::min(std::max(y[i], 0.5f), (float)s.ny - 1.5f);
        int col = (int)std::min(px - 0.5f, (float)(s.nx - 3));
        int row = (int)std::min(py - 0.5f, (float)(s.ny - 3));
        uint8_t& b = seen[(size_t)row * cols + col];
        if (!b) {
            b = 1;
            occupied++;
        }
    }
    return occupied ? (double)s.particles / occupied : 1.0;
}

struct Particles {
    const float *x, *y, *u, *v, *m;
    std::vector<int64_t> first;   // first particle of each scene
};

// Times whole steps of the given scenes with their tile choices and a block size; returns us per step.
int32_t time_batch(const std::vector<vf_scene2>& all, const std::vector<int>& pick, uint32_t flags, int block,
                   const Particles& P, double* us) {
    std::vector<vf_scene2> sc;
    std::vector<float> f[5];
    for (int s : pick) {
        sc.push_back(all[s]);
        const float* src[5] = {P.x, P.y, P.u, P.v, P.m};
        for (int k = 0; k < 5; k++)
            f[k].insert(f[k].end(), src[k] + P.first[s], src[k] + P.first[s] + all[s].particles);
    }
    vf_mpm2_batch* h = nullptr;
    int32_t rc = vf_mpm2_batch_create(sc.data(), (int)sc.size(), flags, block, &h);
    if (rc) return rc;
    void *e0 = nullptr, *e1 = nullptr;
    float ms = 0;
    if ((rc = vf_mpm2_batch_load(h, f[0].data(), f[1].data(), f[2].data(), f[3].data(), f[4].data())) ||
        (rc = vf_mpm2_batch_advance(h, WARM_STEPS)) || (rc = vf_mpm2_batch_finish(h)) ||
        (rc = vf_event_create(&e0)) || (rc = vf_event_create(&e1)) ||
        (rc = vf_event_record(e0, vf_mpm2_batch_stream(h))) || (rc = vf_mpm2_batch_advance(h, TIMED_STEPS)) ||
        (rc = vf_event_record(e1, vf_mpm2_batch_stream(h))) || (rc = vf_event_elapsed_ms(e0, e1, &ms)) ||
        (rc = vf_mpm2_batch_finish(h))) {
    }
    if (e0) vf_event_destroy(e0);
    if (e1) vf_event_destroy(e1);
    vf_mpm2_batch_destroy(h);
    *us = 1000.0 * ms / TIMED_STEPS;
    return rc;
}

}  // namespace

extern "C" int32_t vf_mpm2_autotune(vf_scene2* scenes, int32_t nscenes, uint32_t flags, const float* x,
                                    const float* y, const float* u, const float* v, const float* m,
                                    const char* cache_path, int32_t* block, int32_t* trials) {
    VF_REQUIRE(scenes && nscenes >= 1 && x && y && u && v && m && block, VF_EINVAL, "null or empty argument");
    int32_t rc = require_device();
    if (rc) return rc;
    int dev = 0;
    cudaDeviceProp prop;
    VF_TRY_CUDA(cudaGetDevice(&dev));
    VF_TRY_CUDA(cudaGetDeviceProperties(&prop, dev));
    const std::string device = prop.name;
    Particles P{x, y, u, v, m, {}};
    int64_t at = 0;
    std::vector<std::pair<int, int>> key((size_t)nscenes);
    std::map<std::pair<int, int>, std::vector<int>> members;
    for (int s = 0; s < nscenes; s++) {
        VF_REQUIRE(scenes[s].nx >= 3 && scenes[s].ny >= 3 && scenes[s].particles >= 1, VF_EINVAL,
                   "scene %d: nx, ny >= 3 and particles >= 1", s);
        P.first.push_back(at);
        key[s] = {pow2_round(scene_ppc(scenes[s], x + at, y + at)), pow2_up(std::max(scenes[s].nx, scenes[s].ny))};
        members[key[s]].push_back(s);
        at += scenes[s].particles;
    }
    Cache cache = read_cache(cache_path);
    int ran = 0;
    // 1. tile shape per key
    std::map<std::pair<int, int>, std::pair<int, int>> tile;
    for (auto& kv : members) {
        for (const TileEntry& e : cache.tiles)
            if (e.device == device && e.ppc == kv.first.first && e.n == kv.first.second) tile[kv.first] = {e.tx, e.ty};
        if (tile.count(kv.first)) continue;
        std::vector<int> pick(kv.second.begin(), kv.second.begin() + std::min<size_t>(kv.second.size(), TUNE_SCENES));
        std::vector<vf_scene2> trial(scenes, scenes + nscenes);
        double best = 1e300;
        std::pair<int, int> choice{16, 16};
        for (auto& t : TILES) {
            for (int s : pick) {
                trial[s].tile_x = t[0];
                trial[s].tile_y = t[1];
            }
            double us = 0;
            if ((rc = time_batch(trial, pick, flags, 256, P, &us))) return rc;
            ran++;
            if (us < best) {
                best = us;
                choice = {t[0], t[1]};
            }
        }
        tile[kv.first] = choice;
        cache.tiles.push_back({device, kv.first.first, kv.first.second, choice.first, choice.second, best});
    }
    for (int s = 0; s < nscenes; s++) {
        scenes[s].tile_x = tile[key[s]].first;
        scenes[s].tile_y = tile[key[s]].second;
    }
    // 2. block size for this batch's key set
    std::string keys;
    for (auto& kv : members) keys += (keys.empty() ? "" : " ") + std::to_string(kv.first.first) + "/" +
                                     std::to_string(kv.first.second);
    int chosen = 0;
    for (const BlockEntry& e : cache.blocks)
        if (e.device == device && e.keys == keys) chosen = e.block;
    if (!chosen) {
        std::vector<int> pick;   // round-robin over the keys
        for (size_t r = 0; (int)pick.size() < std::min(nscenes, BLOCK_SCENES); r++)
            for (auto& kv : members)
                if (r < kv.second.size() && (int)pick.size() < BLOCK_SCENES) pick.push_back(kv.second[r]);
        std::vector<vf_scene2> trial(scenes, scenes + nscenes);
        double best = 1e300;
        for (int b : BLOCKS) {
            double us = 0;
            if ((rc = time_batch(trial, pick, flags, b, P, &us))) return rc;
            ran++;
            if (us < best) {
                best = us;
                chosen = b;
            }
        }
        cache.blocks.push_back({device, keys, chosen, best});
    }
    *block = chosen;
    if (trials) *trials = ran;
    return ran ? write_cache(cache_path, cache) : VF_OK;
}
