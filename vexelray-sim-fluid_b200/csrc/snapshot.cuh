// snapshot.cuh -- the versioned binary snapshot of a simulation's state, for replay, resume and cross-run
// parity (no counterpart in the reference, which has only load() and readbacks).
//
// Layout (little-endian): a 64-byte header, then the kind's payload. The header names the kind, the sizes the
// payload was taken at, the step count, and the payload's length and FNV-1a 64 checksum; a restore refuses a
// snapshot whose magic, version, kind, sizes, length or checksum differ from what the handle expects.
//   kind 3, 3D MLS-MPM: 7 param words (Flip3.params: dt, gx, gy, gz, bulk, rho0, sigma as float bits), the 17
//     particle fields of the current set (x y z u v w m j c00..c22, each np floats, in the set's order), the last
//     scatter's grid (nodes float4 {m, mu, mv, mw}).
//   kind 2, shallow water: 5 param words, the host clock, the dispatch count and the last step's ticks (3 int64),
//     the current speed word, budget word and clamp count (3 int32), then h, hu, hv (cells floats each).
#pragma once

#include "common.cuh"

namespace vf {

enum : uint32_t { SNAP_VERSION = 1, SNAP_SWE = 2, SNAP_MPM3 = 3 };

struct SnapHeader {
    char magic[8];        // "VFSNAP\0\0"
    uint32_t version;     // SNAP_VERSION
    uint32_t kind;        // SNAP_*
    int32_t nx, ny, nz;
    int32_t flags;        // the physics flags (3D) or the four edges, 8 bits each (shallow water)
    int64_t count;        // particles or cells
    int64_t steps;
    uint64_t payload;     // bytes after the header
    uint64_t checksum;    // FNV-1a 64 of the payload
};
static_assert(sizeof(SnapHeader) == 64, "the snapshot header is 64 bytes");

inline uint64_t fnv1a(const void* data, size_t n, uint64_t h = 1469598103934665603ull) {
    const unsigned char* p = static_cast<const unsigned char*>(data);
    for (size_t i = 0; i < n; i++) {
        h ^= p[i];
        h *= 1099511628211ull;
    }
    return h;
}

inline SnapHeader snap_header(uint32_t kind, int nx, int ny, int nz, int32_t flags, int64_t count, int64_t steps,
                              uint64_t payload) {
    SnapHeader hd{};
    memcpy(hd.magic, "VFSNAP\0\0", 8);
    hd.version = SNAP_VERSION;
    hd.kind = kind;
    hd.nx = nx;
    hd.ny = ny;
    hd.nz = nz;
    hd.flags = flags;
    hd.count = count;
    hd.steps = steps;
    hd.payload = payload;
    return hd;
}

// Checks a snapshot against what a handle expects; VF_EINVAL with the first difference.
inline int32_t snap_check(const void* buf, int64_t size, const SnapHeader& want, SnapHeader* got) {
    VF_REQUIRE(buf && size >= (int64_t)sizeof(SnapHeader), VF_EINVAL, "a snapshot has a 64-byte header, got %lld bytes",
               (long long)size);
    memcpy(got, buf, sizeof(SnapHeader));
    VF_REQUIRE(memcmp(got->magic, "VFSNAP\0\0", 8) == 0, VF_EINVAL, "not a snapshot (magic)");
    VF_REQUIRE(got->version == SNAP_VERSION, VF_EINVAL, "snapshot version %u, this library reads %u", got->version,
               SNAP_VERSION);
    VF_REQUIRE(got->kind == want.kind, VF_EINVAL, "a snapshot of kind %u, this handle takes kind %u", got->kind, want.kind);
    VF_REQUIRE(got->nx == want.nx && got->ny == want.ny && got->nz == want.nz && got->count == want.count, VF_EINVAL,
               "a snapshot of %d x %d x %d with %lld elements, this handle is %d x %d x %d with %lld", got->nx, got->ny,
               got->nz, (long long)got->count, want.nx, want.ny, want.nz, (long long)want.count);
    VF_REQUIRE(got->flags == want.flags, VF_EINVAL, "a snapshot taken with flags 0x%x, this handle has 0x%x", got->flags,
               want.flags);
    VF_REQUIRE(got->payload == want.payload && (int64_t)(sizeof(SnapHeader) + got->payload) == size, VF_EINVAL,
               "a snapshot payload of %llu bytes in %lld, expected %llu", (unsigned long long)got->payload,
               (long long)size, (unsigned long long)want.payload);
    VF_REQUIRE(fnv1a(static_cast<const char*>(buf) + sizeof(SnapHeader), got->payload) == got->checksum, VF_EINVAL,
               "the snapshot's checksum does not match its payload");
    return VF_OK;
}

}  // namespace vf
