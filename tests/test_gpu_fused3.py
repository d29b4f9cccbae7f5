"""The fused 3D step (k_g2p2g3: the gather of step k and the scatter of step k+1 in one kernel) against the oracle's
Flip3Step (Flip3.java:193-383), and against the separate tiled passes.

Parity bars (tolerances written here, the same as the other 3D schedules'):
* grid mass and momentum after k steps: per node |gpu - oracle| <= 1e-5 * max(1, |oracle|); after two or more steps
  the grid the readout shows is the fused kernel's own scatter;
* particle positions after many steps: |gpu - oracle| <= 1e-4 * |oracle| per coordinate, particles matched by
  their masses (each particle's mass made distinct by one ulp per particle);
* total mass: the particles' masses are the same multiset, bit for bit.
The scenes throw particles across cells every step, so the kernel's movers (particles that leave their sorted cell)
go through both of its paths: into the unit's window, and straight into the grid when they leave it.
"""
import math

import numpy as np
import pytest

import vexfluid as vf
from _oracle import F, Flip3State, flip3_params

pytestmark = pytest.mark.gpu


def tagged(m):
    return (np.asarray(m, F).view(np.int32) + np.arange(len(m), dtype=np.int32)).view(F)


def stirred(n=40, count=30000, speed=25.0, seed=3):
    """Particles in [4, n-4)^3 with random velocities of up to `speed` nodes/s: at dt = 0.01 a quarter of a cell a
    step, so every step moves a good share of them into another cell (and some across units and bricks)."""
    r = np.random.default_rng(seed)
    pos = (4 + r.random((3, count)) * (n - 8)).astype(F)
    vel = r.uniform(-speed, speed, (3, count)).astype(F)
    m = tagged(np.full(count, 0.125, F))
    return pos, vel, m, (0.01, 0.0, -10.0, 0.0, 400.0, 1.0)


def check_grid(grid, o, what):
    for f, key in enumerate(("gm", "gmu", "gmv", "gmw")):
        e = o.g[key].astype(np.float64)
        err = np.abs(grid[f] - e)
        bad = err > 1e-5 * np.maximum(1, np.abs(e))
        assert not bad.any(), (what, key, int(bad.sum()), float(err.max()))


def check_positions(s, o, what):
    pos = s.positions()
    mass = s.read("m")
    dev = np.argsort(mass.view(np.int32))
    ora = np.argsort(o.a["m"].view(np.int32))
    assert np.array_equal(mass.view(np.int32)[dev], o.a["m"].view(np.int32)[ora]), what
    for a, key in enumerate(("x", "y", "z")):
        e = o.a[key][ora]
        err = np.abs(pos[a][dev] - e)
        assert np.all(err <= 1e-4 * np.abs(e)), (what, key, float((err / np.abs(e)).max()))


def test_fused_is_an_option_of_the_sorted_tile():
    pos, vel, m, p = stirred(count=1000)
    with vf.ParticleSimulation3(40, 40, 40, len(m)) as s:
        assert not s.fused()
        s.set_fused(True)
        assert s.fused()
        s.set_fused(False)
        assert not s.fused()
    with vf.ParticleSimulation3(40, 40, 40, len(m), schedule=vf.VF_P2G_ATOMIC) as s:
        assert not s.fused()


@pytest.mark.parametrize("steps", [2, 3, 6])
def test_fused_scatter_matches_the_oracle_per_node(steps):
    """After two or more steps the grid shown is the fused kernel's scatter of the particles it just moved."""
    n = 40
    pos, vel, m, p = stirred(n)
    o = Flip3State(n, n, n, *pos, m, u=vel[0], v=vel[1], w=vel[2])
    with vf.ParticleSimulation3(n, n, n, len(m)) as s:
        s.set_fused(True)
        assert s.fused()
        s.load(list(pos), list(vel), m, vf.flip3_params(*p))
        s.advance(steps)
        for _ in range(steps):
            o.step(flip3_params(*p))
        check_grid(s.grid(), o, f"after {steps} steps")
        check_positions(s, o, f"after {steps} steps")


def test_fused_positions_after_forty_steps_match_the_oracle_and_the_separate_passes():
    n = 40
    pos, vel, m, p = stirred(n, count=20000, speed=15.0, seed=5)
    o = Flip3State(n, n, n, *pos, m, u=vel[0], v=vel[1], w=vel[2])
    for _ in range(40):
        o.step(flip3_params(*p))
    for fused in (True, False):
        with vf.ParticleSimulation3(n, n, n, len(m)) as s:
            s.set_fused(fused)
            s.load(list(pos), list(vel), m, vf.flip3_params(*p))
            s.advance(40)
            check_positions(s, o, f"fused={fused}")
            check_grid(s.grid(), o, f"fused={fused}")
            assert np.array_equal(np.sort(s.read("m").view(np.int32)), np.sort(m.view(np.int32)))


def test_calls_between_fused_steps_see_and_keep_the_reference_state():
    """The fused step scatters the next step early; params changes, field writes, readouts, snapshots and passes
    run on their own all see (or discard) it so the run stays the oracle's."""
    n = 40
    pos, vel, m, p = stirred(n, count=12000, seed=9)
    o = Flip3State(n, n, n, *pos, m, u=vel[0], v=vel[1], w=vel[2])
    p2 = (0.008, 0.0, -20.0, 0.0, 600.0, 1.0)
    with vf.ParticleSimulation3(n, n, n, len(m)) as s:
        s.set_fused(True)
        s.load(list(pos), list(vel), m, vf.flip3_params(*p))
        s.advance(3)
        for _ in range(3):
            o.step(flip3_params(*p))
        check_grid(s.grid(), o, "3 steps")
        # new params: the early scatter (made with the old ones) must not be used
        s.params(vf.flip3_params(*p2))
        s.advance(2)
        for _ in range(2):
            o.step(flip3_params(*p2))
        check_grid(s.grid(), o, "2 steps with new params")
        check_positions(s, o, "2 steps with new params")
        # a write of a velocity field between steps
        u = s.read("u")
        mass = s.read("m")
        u2 = (u * np.float32(0.5)).astype(F)
        s.write("u", u2)
        ora = np.argsort(o.a["m"].view(np.int32))
        dev = np.argsort(mass.view(np.int32))
        o.a["u"][ora] = u2[dev]
        s.advance(2)
        for _ in range(2):
            o.step(flip3_params(*p2))
        check_grid(s.grid(), o, "after a write")
        check_positions(s, o, "after a write")
        # a snapshot mid-run restores into a new handle and continues the same
        blob = s.snapshot()
        s.advance(3)
        with vf.ParticleSimulation3(n, n, n, len(m)) as t:
            t.set_fused(True)
            t.restore(blob)
            t.advance(3)
            a, b = s.positions(), t.positions()
            ma, mb = s.read("m"), t.read("m")
            ia, ib = np.argsort(ma.view(np.int32)), np.argsort(mb.view(np.int32))
            for k in range(3):
                assert np.all(np.abs(a[k][ia] - b[k][ib]) <= 1e-4 * np.abs(a[k][ia]))


def test_a_unit_holding_more_than_the_staged_particles():
    """A column compressed to 48 particles a cell: an 8 x 8 x 1 unit of cells holds over 2,048 particles, more than
    the tiled scatter stages in shared memory, so its cells' runs are put in order in place. The first scatter (the
    tiled one), the fused steps after it and the separate passes all stay within the oracle's bars."""
    n = 32
    r = np.random.default_rng(17)
    # stencil cells 8..15 x 8..15 x 8..9 (one brick's two lowest 8 x 8 x 1 units), 48 particles each
    cells = np.argwhere(np.ones((8, 8, 2), bool)).astype(F) + np.array([8.5, 8.5, 8.5], F)
    per = 48
    pos = (np.repeat(cells, per, axis=0) + r.random((len(cells) * per, 3), dtype=np.float32) * np.float32(0.999))
    x, y, z = (np.ascontiguousarray(pos[:, a], F) for a in range(3))
    m = tagged(np.full(len(x), 0.02, F))
    assert len(x) == 2 * 64 * per and 64 * per > 2048
    p = (0.002, 0.0, -10.0, 0.0, 100.0, 1.0)
    for fused in (True, False):
        o = Flip3State(n, n, n, x, y, z, m)
        with vf.ParticleSimulation3(n, n, n, len(x)) as s:
            s.set_fused(fused)
            s.load([x, y, z], [np.zeros_like(x)] * 3, m, vf.flip3_params(*p))
            for k in range(1, 4):
                s.advance(1)
                o.step(flip3_params(*p))
                check_grid(s.grid(), o, f"fused={fused} step {k}")
            check_positions(s, o, f"fused={fused}")
