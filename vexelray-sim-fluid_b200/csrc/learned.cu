// learned.cu -- the learned coarse shallow-water solver's driver as a native handle (vf_swe_learned_*): a coarse
// patch stepped by the plain HLL step, the flux-correction network's correction applied once an interval, and
// tiles whose relative depth jump crosses a threshold stepped by the fine solver instead. No counterpart in the
// reference; its error is measured against the plain fine solver (ShallowWater.kernel, ShallowWater.java:166-242).
//
// One interval of `interval` ticks:
//   [fallback]  the coarse state's per-tile jump (vf_swe_jump_indicator); if any tile trips, the state is kept
//   predict     the network's correction from the interval's start state, on the coarse stream
//   advance     the coarse patch through the interval (vf_swe_advance)
//   apply       the correction added at the interval's end, and the coarse wave speed measured
//   [fallback]  each tripped tile, with a margin, prolonged from the kept state into a fine patch, stepped through
//               the interval and restricted back into the coarse state; the wave speed measured again
#include <cmath>
#include <cstring>
#include <map>
#include <tuple>
#include <vector>

#include "common.cuh"

namespace {

constexpr float G = 9.81f, COURANT = 0.45f, DRY = 1e-6f;
constexpr int32_t NEVER = 2147483647;   // a step budget that does not stop the steps
// Coarse steps an interval may take before the driver gives up on it (about 64 times the usual 16): a state a
// correction has driven toward dry or violent flow shrinks the step toward a tick and would otherwise spin. The
// reference's test stepper stops a run the same way when its steps stop growing
// (vexelray-sim-fluid-core/src/test/java/dev/vexelray/sim/fluid/stencil/Stepper.java:90-93).
constexpr int32_t INTERVAL_STEP_CAP = 1024;

void swe_words(float dx, int32_t out[5]) {
    const float w[5] = {G, COURANT, dx, dx, DRY};
    memcpy(out, w, sizeof w);
}

// A state at rest with unit depth (the fine patches and the kept start state are overwritten before use).
int32_t load_rest(vf_swe* s, int nx, int ny, float dx) {
    std::vector<float> one((size_t)nx * ny, 1.0f), zero((size_t)nx * ny, 0.0f);
    int32_t words[5];
    swe_words(dx, words);
    return vf_swe_load(s, one.data(), zero.data(), zero.data(), words, 5);
}

}  // namespace

struct vf_swe_learned {
    int nx = 0, ny = 0, tile = 64, margin = 8;
    float threshold = 0.0f;    // tiles whose jump exceeds it fall back, when `start` exists
    float dx = 1.0f;
    int64_t interval = 0;
    vf_cnn* net = nullptr;     // borrowed; null: the plain coarse solver
    vf_swe* coarse = nullptr;
    vf_swe* start = nullptr;   // the interval's start state, kept when a tile trips
    std::map<std::tuple<int, int, int>, vf_swe*> patches;   // fine patches by (width, height, edges)
    std::vector<float> jump;
    int64_t steps = 0, corrections = 0, fallback_tiles = 0;
};

namespace {

int32_t fine_tile(vf_swe_learned* h, int tx, int ty, int64_t t) {
    const int T = h->tile, m = h->margin;
    const int x0 = tx * T, y0 = ty * T;
    const int w = std::min(T, h->nx - x0), hgt = std::min(T, h->ny - y0);
    const int bx0 = std::max(0, x0 - m), by0 = std::max(0, y0 - m);
    const int bx1 = std::min(h->nx, x0 + w + m), by1 = std::min(h->ny, y0 + hgt + m);
    const int32_t edges[4] = {bx0 == 0 ? VF_EDGE_WALL : VF_EDGE_OPEN, bx1 == h->nx ? VF_EDGE_WALL : VF_EDGE_OPEN,
                              by0 == 0 ? VF_EDGE_WALL : VF_EDGE_OPEN, by1 == h->ny ? VF_EDGE_WALL : VF_EDGE_OPEN};
    const auto key = std::make_tuple(bx1 - bx0, by1 - by0, edges[0] | edges[1] << 1 | edges[2] << 2 | edges[3] << 3);
    vf_swe* patch;
    auto it = h->patches.find(key);
    if (it == h->patches.end()) {
        int32_t rc = vf_swe_create(2 * (bx1 - bx0), 2 * (by1 - by0), edges, &patch);
        if (rc) return rc;
        h->patches[key] = patch;
        if ((rc = load_rest(patch, 2 * (bx1 - bx0), 2 * (by1 - by0), h->dx))) return rc;
    } else {
        patch = it->second;
    }
    int32_t rc = vf_swe_prolong(h->start, bx0, by0, patch);
    if (!rc) rc = vf_swe_advance(patch, t, NEVER, nullptr, nullptr, nullptr);
    if (!rc) rc = vf_swe_restrict_patch(patch, 2 * (x0 - bx0), 2 * (y0 - by0), h->coarse, x0, y0, w, hgt);
    if (!rc) h->fallback_tiles++;
    return rc;
}

}  // namespace

extern "C" {

int32_t vf_swe_learned_create(int32_t nx, int32_t ny, vf_cnn* net, int64_t interval_ticks, int32_t tile,
                              int32_t fallback, float threshold, int32_t margin, float dx, vf_swe_learned** out) {
    VF_REQUIRE(out, VF_EINVAL, "out is null");
    *out = nullptr;
    VF_REQUIRE(interval_ticks >= 1, VF_EINVAL, "an interval is at least one tick, got %lld", (long long)interval_ticks);
    VF_REQUIRE(tile >= 1 && margin >= 0 && dx > 0, VF_EINVAL, "tile >= 1, margin >= 0 and dx > 0, got %d, %d, %g", tile,
               margin, dx);
    vf_swe_learned* h = new vf_swe_learned();
    h->nx = nx;
    h->ny = ny;
    h->net = net;
    h->interval = interval_ticks;
    h->tile = tile;
    h->threshold = threshold;
    h->margin = margin;
    h->dx = dx;
    const int32_t walls[4] = {VF_EDGE_WALL, VF_EDGE_WALL, VF_EDGE_WALL, VF_EDGE_WALL};
    int32_t rc = vf_swe_create(nx, ny, walls, &h->coarse);
    if (!rc && fallback) rc = vf_swe_create(nx, ny, walls, &h->start);
    if (!rc && h->start) rc = load_rest(h->start, nx, ny, 2 * dx);
    if (rc) {
        vf_swe_learned_destroy(h);
        return rc;
    }
    h->jump.resize((size_t)((nx + tile - 1) / tile) * ((ny + tile - 1) / tile));
    *out = h;
    return VF_OK;
}

int32_t vf_swe_learned_load(vf_swe_learned* h, const float* hcell, const float* hu, const float* hv) {
    VF_REQUIRE(h && hcell && hu && hv, VF_EINVAL, "null argument");
    int32_t words[5];
    swe_words(2 * h->dx, words);
    return vf_swe_load(h->coarse, hcell, hu, hv, words, 5);
}

int32_t vf_swe_learned_advance(vf_swe_learned* h, int64_t ticks) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    VF_REQUIRE(ticks >= 0, VF_EINVAL, "ticks must be >= 0");
    const int ntx = (h->nx + h->tile - 1) / h->tile;
    for (int64_t left = ticks; left > 0;) {
        const int64_t t = std::min(h->interval, left);
        std::vector<std::pair<int, int>> tripped;
        int32_t rc;
        if (h->start) {
            if ((rc = vf_swe_jump_indicator(h->coarse, h->tile, h->jump.data(), (int32_t)h->jump.size()))) return rc;
            for (size_t k = 0; k < h->jump.size(); k++)   // row-major: tiles of a row by x, rows by y
                if (h->jump[k] > h->threshold) tripped.emplace_back((int)(k % ntx), (int)(k / ntx));
            if (!tripped.empty() && (rc = vf_swe_copy_state(h->start, h->coarse))) return rc;
        }
        float *sh, *su, *sv;
        if (h->net) {
            if ((rc = vf_swe_state(h->coarse, &sh, &su, &sv))) return rc;
            if ((rc = vf_cnn_predict(h->net, sh, su, sv, vf_swe_stream(h->coarse)))) return rc;
        }
        int32_t steps = 0;
        int64_t spent = 0;
        if ((rc = vf_swe_advance(h->coarse, t, INTERVAL_STEP_CAP, &steps, &spent, nullptr))) return rc;
        h->steps += steps;
        VF_REQUIRE(spent >= t, VF_ESTATE,
                   "the corrected coarse state stopped advancing: %d steps covered %lld of the interval's %lld ticks "
                   "(correction %lld)", steps, (long long)spent, (long long)t, (long long)h->corrections);
        if (h->net) {
            if ((rc = vf_swe_state(h->coarse, &sh, &su, &sv))) return rc;
            if ((rc = vf_cnn_apply(h->net, sh, su, sv, vf_swe_stream(h->coarse)))) return rc;
            if ((rc = vf_swe_measure_speed(h->coarse))) return rc;
            h->corrections++;
        }
        for (const auto& tt : tripped)
            if ((rc = fine_tile(h, tt.first, tt.second, t))) return rc;
        if (!tripped.empty() && (rc = vf_swe_measure_speed(h->coarse))) return rc;
        left -= t;
    }
    return VF_OK;
}

int32_t vf_swe_learned_read(vf_swe_learned* h, float* hcell, float* hu, float* hv) {
    VF_REQUIRE(h, VF_EINVAL, "null handle");
    return vf_swe_read(h->coarse, hcell, hu, hv);
}

int32_t vf_swe_learned_counts(const vf_swe_learned* h, int64_t out[3]) {
    VF_REQUIRE(h && out, VF_EINVAL, "null argument");
    out[0] = h->steps;
    out[1] = h->corrections;
    out[2] = h->fallback_tiles;
    return VF_OK;
}

vf_swe* vf_swe_learned_coarse(vf_swe_learned* h) { return h ? h->coarse : nullptr; }

void vf_swe_learned_destroy(vf_swe_learned* h) {
    if (!h) return;
    for (auto& kv : h->patches) vf_swe_destroy(kv.second);
    vf_swe_destroy(h->start);
    vf_swe_destroy(h->coarse);
    delete h;
}

}  // extern "C"
