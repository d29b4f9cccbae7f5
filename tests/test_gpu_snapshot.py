"""Snapshots of the 3D simulation and the shallow-water patch: a restored run resumes bit for bit, and a snapshot
that does not fit the handle, or whose payload was changed, is refused.

Parity bar: bit-exact. The 3D run uses the exact scatter schedule (VF_P2G_FIXED), under which a whole step is
deterministic (stable sort, integer sums, per-particle gather); the shallow-water step is bit-exact anyway.
"""
import struct

import numpy as np
import pytest

import vexfluid as vf
from _oracle import F, swe_params
from test_gpu_mpm3 import dam3
from test_gpu_swe import bumps

pytestmark = pytest.mark.gpu

FIELDS3 = ["x", "y", "z", "u", "v", "w", "m", "j"] + [f"c{a}{b}" for a in range(3) for b in range(3)]


def fnv1a64(data: bytes) -> int:
    h = 1469598103934665603
    for b in data:
        h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def header(blob: bytes) -> dict:
    magic, version, kind, nx, ny, nz, flags, count, steps, payload, checksum = struct.unpack("<8s2I4i2q2Q", blob[:64])
    return dict(magic=magic, version=version, kind=kind, dims=(nx, ny, nz), flags=flags, count=count, steps=steps,
                payload=payload, checksum=checksum)


def state3(s):
    return [s.read(f).view(np.int32).copy() for f in FIELDS3], [g.view(np.int32).copy() for g in s.grid()]


def load3(s, x, y, z, m, p):
    s.load([x, y, z], [np.zeros_like(x)] * 3, m, vf.flip3_params(*p))


def test_a_restored_3d_run_continues_bit_for_bit():
    n = 24
    x, y, z, m, p, _ = dam3(n, tagged=True)
    with vf.ParticleSimulation3(n, n, n, len(x), schedule=vf.VF_P2G_FIXED) as a:
        load3(a, x, y, z, m, p)
        a.advance(10)
        blob = a.snapshot()
        at_snapshot = state3(a)
        a.advance(10)
        want = state3(a)
        assert a.steps() == 20
    hd = header(blob)
    assert hd["magic"] == b"VFSNAP\0\0" and hd["version"] == 1 and hd["kind"] == 3
    assert hd["dims"] == (n, n, n) and hd["count"] == len(x) and hd["steps"] == 10
    assert hd["payload"] == len(blob) - 64 == 32 + 17 * len(x) * 4 + n * n * n * 16
    assert hd["checksum"] == fnv1a64(blob[64:])
    # the payload's particle block is the fields in order
    body = np.frombuffer(blob, np.int32, count=17 * len(x), offset=64 + 32).reshape(17, len(x))
    for f in range(17):
        assert np.array_equal(body[f], at_snapshot[0][f]), FIELDS3[f]
    with vf.ParticleSimulation3(n, n, n, len(x), schedule=vf.VF_P2G_FIXED) as b:
        b.restore(blob)
        assert b.steps() == 10
        fields, grid = state3(b)
        for f in range(17):
            assert np.array_equal(fields[f], at_snapshot[0][f]), FIELDS3[f]
        for g in range(4):
            assert np.array_equal(grid[g], at_snapshot[1][g]), g
        b.advance(10)
        got = state3(b)
        assert b.steps() == 20
    for f in range(17):
        assert np.array_equal(got[0][f], want[0][f]), FIELDS3[f]
    for g in range(4):
        assert np.array_equal(got[1][g], want[1][g]), g


def test_a_3d_snapshot_resumes_under_another_schedule():
    """The tiled schedule's run, restored into the exact schedule and back: the particles and the last grid come
    back as they were, and the run goes on conserving mass to the bit."""
    n = 24
    x, y, z, m, p, _ = dam3(n, tagged=True)
    with vf.ParticleSimulation3(n, n, n, len(x)) as a:
        load3(a, x, y, z, m, p)
        a.advance(5)
        blob = a.snapshot()
        before = state3(a)
    for schedule in (vf.VF_P2G_FIXED, vf.VF_P2G_TILE, vf.VF_P2G_ATOMIC):
        with vf.ParticleSimulation3(n, n, n, len(x), schedule=schedule) as b:
            b.restore(blob)
            fields, grid = state3(b)
            assert all(np.array_equal(fields[f], before[0][f]) for f in range(17))
            assert all(np.array_equal(grid[g], before[1][g]) for g in range(4))
            b.advance(5)
            assert b.steps() == 10
            assert np.array_equal(np.sort(b.read("m").view(np.int32)), np.sort(m.view(np.int32)))


def test_a_snapshot_that_does_not_fit_is_refused():
    n = 16
    x, y, z, m, p, _ = dam3(n)
    with vf.ParticleSimulation3(n, n, n, len(x)) as a:
        load3(a, x, y, z, m, p)
        a.advance(2)
        blob = a.snapshot()
    with vf.ParticleSimulation3(n, n, n, len(x)) as b:
        for bad in (blob[:63], blob[:-4], blob + b"\0" * 4):
            with pytest.raises(ValueError):
                b.restore(bad)
        flipped = bytearray(blob)
        flipped[64 + 32 + 5] ^= 1
        with pytest.raises(ValueError, match="checksum"):
            b.restore(bytes(flipped))
        wrong_magic = b"XXSNAP\0\0" + blob[8:]
        with pytest.raises(ValueError, match="magic"):
            b.restore(wrong_magic)
        newer = blob[:8] + struct.pack("<I", 2) + blob[12:]
        with pytest.raises(ValueError, match="version"):
            b.restore(newer)
        # nothing was changed by the refusals: the good blob still restores
        b.restore(blob)
        assert b.steps() == 2
    with vf.ParticleSimulation3(n + 1, n, n, len(x)) as c:
        with pytest.raises(ValueError):
            c.restore(blob)
    with vf.ParticleSimulation3(n, n, n, len(x), tait=True) as d:
        with pytest.raises(ValueError, match="flags"):
            d.restore(blob)
    with vf.PatchSimulation(n, n) as e:
        with pytest.raises(ValueError, match="kind"):
            e.restore(blob)


def swe_state(p):
    return [f.view(np.int32).copy() for f in p.read()], p.now(), p.steps(), p.fastest_wave(), p.clamped()


def test_a_restored_patch_resumes_bit_for_bit():
    n = 96
    h = bumps(n, 5)
    z = np.zeros(n * n, F)
    params = swe_params(9.81, 0.45, 1, 1, 1e-6).view(np.int32)
    edges = (0, 1, 1, 0)
    later = [(vf.ticks(0.05), 1000), (vf.ticks(0.2), 7), (0, 3), (vf.ticks(0.5), 1000)]
    with vf.PatchSimulation(n, n, edges) as a:
        a.load(h, z, z, params)
        a.advance(vf.ticks(0.1), 1000)
        a.advance(vf.ticks(0.1), 3)
        blob = a.snapshot()
        at_snapshot = swe_state(a)
        records = [(r.steps, r.spent_ticks, r.behind_ticks) for r in (a.advance(t, k) for t, k in later)]
        want = swe_state(a)
    hd = header(blob)
    assert hd["kind"] == 2 and hd["dims"] == (n, n, 1) and hd["count"] == n * n
    assert hd["flags"] == edges[0] | edges[1] << 8 | edges[2] << 16 | edges[3] << 24
    assert hd["steps"] == at_snapshot[2] and hd["checksum"] == fnv1a64(blob[64:])
    with vf.PatchSimulation(n, n, edges) as b:
        b.restore(blob)
        got0 = swe_state(b)
        assert all(np.array_equal(got0[0][f], at_snapshot[0][f]) for f in range(3))
        assert got0[1:] == at_snapshot[1:]
        got_records = [(r.steps, r.spent_ticks, r.behind_ticks) for r in (b.advance(t, k) for t, k in later)]
        got = swe_state(b)
    assert got_records == records
    assert all(np.array_equal(got[0][f], want[0][f]) for f in range(3))
    assert got[1:] == want[1:]
    with vf.PatchSimulation(n, n, (0, 0, 0, 0)) as c:
        with pytest.raises(ValueError, match="flags"):
            c.restore(blob)
    with vf.PatchSimulation(n, n - 1, edges) as d:
        with pytest.raises(ValueError):
            d.restore(blob)
