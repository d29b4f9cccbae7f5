"""Batched 2D scenes on the GPU: every scene of a batch against the oracle stepping that scene alone
(FlipStep.step: clear, scatter, grid, advect).

Parity bars (tolerances written here):
* grid mass and momentum after one step: per node |gpu - oracle| <= 1e-5 * max(1, |oracle|);
* particle positions after 100 steps: |gpu - oracle| <= 1e-4 * |oracle| per coordinate, particles matched by
  their masses (each scene's masses are made distinct by one ulp per particle);
* total mass: each scene's masses are the same multiset, bit for bit, after any number of steps.
"""
import json

import numpy as np
import pytest

import bench
import vexfluid as vf
from _oracle import F, Flip2State

pytestmark = pytest.mark.gpu

# (nx, ny, particles): uneven grids and counts, small enough for the oracle
SHAPES = [(32, 40, 700), (48, 48, 2500), (64, 64, 3000), (100, 60, 5000), (70, 90, 1500), (130, 50, 9000)]


def tagged(m):
    """Masses made distinct: the k-th particle's mass k ulps above the base."""
    bits = np.asarray(m, F).view(np.int32) + np.arange(len(m), dtype=np.int32)
    return bits.view(F)


def make_batch(seed, physics, shapes=SHAPES, velocity=2.0):
    rng = np.random.default_rng(seed)
    scenes, parts = [], []
    for k, (nx, ny, count) in enumerate(shapes):
        x, y, m, (dt, gx, gy, bulk, rho0) = bench.dam2_scene(rng, min(nx, ny), count)
        x = np.minimum(x, np.float32(nx - 2))
        y = np.minimum(y, np.float32(ny - 2))
        if physics == "reference":   # p = B(1/J - 1), the wall ring
            bulk = 4e3
        u = rng.uniform(-velocity, velocity, count).astype(F)
        v = rng.uniform(-velocity, velocity, count).astype(F)
        params = vf.flip_params(dt, gx, gy, bulk, rho0)
        tile = vf.BATCH_TILES[k % len(vf.BATCH_TILES)]
        scenes.append(vf.Scene(nx, ny, count, params, tile))
        parts.append((x, y, u, v, tagged(m), (dt, gx, gy, bulk, rho0)))
    return scenes, parts


def flags_of(physics):
    return {"tait": True, "sticky": bench.WALL_BATCH} if physics == "config" else {}


def oracle_physics(physics):
    return (1, bench.WALL_BATCH) if physics == "config" else (0, 0)


def load(b, parts):
    b.load(*[[p[f] for p in parts] for f in range(5)])


def oracle_scene(scene, part):
    x, y, u, v, m, _ = part
    return Flip2State(scene.nx, scene.ny, x, y, m, u=u, v=v)


@pytest.mark.parametrize("physics", ["config", "reference"])
@pytest.mark.parametrize("block", vf.BATCH_BLOCKS)
def test_one_step_grid_matches_the_oracle_per_node(physics, block):
    scenes, parts = make_batch(11, physics)
    with vf.BatchSimulation(scenes, block=block, **flags_of(physics)) as b:
        load(b, parts)
        b.advance(1)
        for k, (sc, p) in enumerate(zip(scenes, parts)):
            o = oracle_scene(sc, p)
            o.step(np.array(p[5], F), oracle_physics(physics))
            for name in ("gm", "gmu", "gmv"):
                got, want = b.read(k, name), o.g[name]
                bad = np.abs(got - want) > 1e-5 * np.maximum(1, np.abs(want))
                assert not bad.any(), (physics, k, name, np.flatnonzero(bad)[:5], got[bad][:5], want[bad][:5])
            assert b.config(k)["tile"] == sc.tile


@pytest.mark.parametrize("physics", ["config", "reference"])
def test_positions_after_100_steps_match_the_oracle(physics):
    scenes, parts = make_batch(12, physics)
    steps = 100
    with vf.BatchSimulation(scenes, **flags_of(physics)) as b:
        load(b, parts)
        b.advance(steps)
        b.finish()
        assert b.steps() == steps
        assert b.launches() == steps + 1   # the load's key tally, then one launch per step
        for k, (sc, p) in enumerate(zip(scenes, parts)):
            o = oracle_scene(sc, p)
            for _ in range(steps):
                o.step(np.array(p[5], F), oracle_physics(physics))
            m = b.read(k, "m")
            # total mass: the same masses, bit for bit
            assert np.array_equal(np.sort(m.view(np.int32)), np.sort(p[4].view(np.int32)))
            order_gpu = np.argsort(m.view(np.int32))
            order_or = np.argsort(o.a["m"].view(np.int32))
            for name in ("x", "y"):
                got = b.read(k, name)[order_gpu]
                want = o.a[name][order_or]
                bad = np.abs(got - want) > 1e-4 * np.abs(want)
                assert not bad.any(), (physics, k, name, np.flatnonzero(bad)[:5], got[bad][:5], want[bad][:5])


def test_particles_stay_in_their_scene_and_in_cell_order():
    """After a step each scene's particles sit at slots sorted by the step's tile-major cell key (the order within
    a cell is left to the atomics, as the reference's CountingSort leaves it). Checked on the positions the step
    started from, the particles matched by their masses."""
    scenes, parts = make_batch(13, "config", velocity=0.5)
    with vf.BatchSimulation(scenes, **flags_of("config")) as b:
        load(b, parts)
        b.advance(3)
        before = [(b.read(k, "x"), b.read(k, "y"), b.read(k, "m")) for k in range(len(scenes))]
        b.advance(1)
        for k, sc in enumerate(scenes):
            x0, y0, m0 = before[k]
            m1 = b.read(k, "m")
            where = {int(v): i for i, v in enumerate(m0.view(np.int32))}
            idx = np.array([where[int(v)] for v in m1.view(np.int32)])
            assert sorted(idx) == list(range(len(idx)))   # the same particles, each once
            px = np.clip(x0[idx], 0.5, sc.nx - 1.5)
            py = np.clip(y0[idx], 0.5, sc.ny - 1.5)
            col = np.minimum(px - np.float32(0.5), sc.nx - 3).astype(np.int64)
            row = np.minimum(py - np.float32(0.5), sc.ny - 3).astype(np.int64)
            tx, ty = sc.tile
            ntx = (sc.nx - 2 + tx - 1) // tx
            key = ((row // ty) * ntx + col // tx) * (tx * ty) + (row % ty) * tx + col % tx
            assert np.all(np.diff(key) >= 0), k


def test_dense_scene_spreads_over_chunks():
    """A 64^2 scene with ~80 particles per cell (tiles of tens of thousands of particles, several work chunks
    each) steps as the oracle does."""
    scenes, parts = make_batch(16, "config", shapes=[(40, 40, 30000), (64, 64, 2000)])
    with vf.BatchSimulation(scenes, **flags_of("config")) as b:
        load(b, parts)
        b.advance(1)
        for k, (sc, p) in enumerate(zip(scenes, parts)):
            o = oracle_scene(sc, p)
            o.step(np.array(p[5], F), oracle_physics("config"))
            for name in ("gm", "gmu", "gmv"):
                got, want = b.read(k, name), o.g[name]
                bad = np.abs(got - want) > 1e-5 * np.maximum(1, np.abs(want))
                assert not bad.any(), (k, name, np.flatnonzero(bad)[:5])


def test_autotune_times_then_reads_its_cache(tmp_path):
    shapes = [(48, 48, 3000), (48, 48, 2000), (100, 60, 600)]
    scenes, parts = make_batch(14, "config", shapes=shapes)
    untuned = [vf.Scene(s.nx, s.ny, s.particles, s.params) for s in scenes]
    cols = [[p[f] for p in parts] for f in range(5)]
    cache = tmp_path / "tune.json"
    tuned, block, trials = vf.autotune(untuned, *cols, cache=cache, **flags_of("config"))
    assert trials >= len(vf.BATCH_TILES) + len(vf.BATCH_BLOCKS)   # at least one key's tiles, then the blocks
    assert block in vf.BATCH_BLOCKS
    assert all(s.tile in vf.BATCH_TILES for s in tuned)
    doc = json.loads(cache.read_text())
    assert doc["entries"] and all("device" in e for e in doc["entries"])
    again, block2, trials2 = vf.autotune(untuned, *cols, cache=cache, **flags_of("config"))
    assert trials2 == 0 and block2 == block and [s.tile for s in again] == [s.tile for s in tuned]
    with vf.BatchSimulation(tuned, block=block, **flags_of("config")) as b:
        load(b, parts)
        b.advance(20)
        b.finish()


def test_refusals():
    scenes, parts = make_batch(15, "config", shapes=[(32, 32, 100)])
    with pytest.raises(vf.IllegalArgumentException):
        vf.BatchSimulation([vf.Scene(32, 32, 100, scenes[0].params, (12, 12))])
    with pytest.raises(vf.IllegalArgumentException):
        vf.BatchSimulation(scenes, block=96)
    with vf.BatchSimulation(scenes) as b:
        with pytest.raises(vf.IllegalStateException):
            b.advance(1)   # nothing loaded
        with pytest.raises(vf.IllegalArgumentException):
            b.load(*[[p[f][:50] for p in parts] for f in range(5)])


def test_a_grid_barrier_that_gives_up_reports_a_timeout():
    """The bounded wait of the step kernel's grid barrier, made to run out: with the poll limit at one, CTAs that
    arrive before the last one give up, set the timeout bit and end the kernel. The next blocking call returns
    VF_ETIMEOUT, the batch refuses to step until it is loaded again, and a reload steps within the oracle's
    one-step bar. (The reference's analogue: Stepper's runaway guard, Stepper.java:88-93.)"""
    scenes, parts = make_batch(13, "config", shapes=SHAPES[:3])
    with vf.BatchSimulation(scenes, **flags_of("config")) as b:
        load(b, parts)
        b.set_wait_limit(1)
        b.advance(1)
        with pytest.raises(vf.VfError) as err:
            b.finish()
        assert err.value.code == vf.VF_ETIMEOUT, err.value
        assert "grid barrier timed out" in str(err.value)
        with pytest.raises(vf.IllegalStateException):
            b.advance(1)
        load(b, parts)   # resets the barrier, the status and the poll limit
        b.advance(1)
        b.finish()
        for k, (sc, p) in enumerate(zip(scenes, parts)):
            o = oracle_scene(sc, p)
            o.step(np.array(p[5], F), oracle_physics("config"))
            for name in ("gm", "gmu", "gmv"):
                got, want = b.read(k, name), o.g[name]
                assert np.all(np.abs(got - want) <= 1e-5 * np.maximum(1, np.abs(want))), (k, name)
    # a fresh batch after the timed-out one was destroyed steps normally
    with vf.BatchSimulation(scenes, **flags_of("config")) as b:
        load(b, parts)
        b.advance(2)
        b.finish()
