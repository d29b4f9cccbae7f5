"""Parity at the configurations' own sizes (the workloads bench.py times), against the oracle.

* 3D dam break, 256^3 nodes, 8,156,736 particles: the sort's starts and particle order bit-exact against the
  oracle's stable counting sort; the grid after one step within 1e-5 * max(1, |oracle|) per node of the oracle's
  threaded step, and after two steps (the fused kernel's own scatter) the same; positions after 20 steps within
  1e-4 relative per coordinate, particles matched by their masses; the masses the same multiset, bit for bit.
* Shallow water, 4096^2 cells, 16 seeded bumps: state, clock and clamp count bit-exact after each of 5 steps.
* Batched 2D scenes, all 256 of the batched configuration (16.1M particles): every scene's grid after one step
  within 1e-5 * max(1, |oracle|) per node of the oracle stepping that scene alone.
These are the sizes where the 24-bit brick-major keys, the 32,768-brick scans and the multi-wave persistent loops
run, so they are checked here and not only on the small cases.
"""
import ctypes

import numpy as np
import pytest

import bench
import vexfluid as vf
from _oracle import (F, Flip2State, Flip3State, OracleSweBackend, OrPhysics, Stepper, flip3_params, fp, lib,
                     swe_params)

pytestmark = pytest.mark.gpu


def dam3_tagged():
    """The 3D configuration with every particle's mass distinct: the k-th float above 1/16 (masses 0.0625 up to
    0.123, all in one binade), so a particle is found by its mass bits through any sort."""
    x, y, z, m, params = bench.dam3()
    m = (np.full(len(x), np.float32(0.0625)).view(np.int32) + np.arange(len(x), dtype=np.int32)).view(F)
    return x, y, z, m, params


def omp_step(o, params):
    lib().or_flip3_step_omp(ctypes.byref(o.s), fp(np.ascontiguousarray(flip3_params(*params), F)), OrPhysics(0, 0),
                            None)


def check_grid3(grid, o, what):
    for f, key in enumerate(("gm", "gmu", "gmv", "gmw")):
        e = o.g[key].astype(np.float64)
        err = np.abs(grid[f] - e)
        bad = err > 1e-5 * np.maximum(1, np.abs(e))
        assert not bad.any(), (what, key, int(bad.sum()), float(err.max()))


def test_3d_configuration_sort_is_bit_exact():
    x, y, z, m, params = dam3_tagged()
    n = bench.N3
    o = Flip3State(n, n, n, x, y, z, m)
    starts_o, _, _ = o.sort()
    with vf.ParticleSimulation3(n, n, n, len(x)) as s:
        s.load([x, y, z], [np.zeros_like(x)] * 3, m, vf.flip3_params(*params))
        s.run(vf.VF3_PASS_SORT)
        assert np.array_equal(s.starts(), starts_o)
        for key in ("x", "y", "z", "m"):
            assert np.array_equal(s.read(key).view(np.int32), o.a[key].view(np.int32)), key


def test_3d_configuration_grid_and_positions_match_the_oracle():
    """The separate tiled passes (the default) and the fused step."""
    x, y, z, m, params = dam3_tagged()
    for fused in (False, True):
        run_3d_configuration(x, y, z, m, params, fused)


def run_3d_configuration(x, y, z, m, params, fused):
    n = bench.N3
    o = Flip3State(n, n, n, x, y, z, m)
    with vf.ParticleSimulation3(n, n, n, len(x)) as s:
        s.set_fused(fused)
        s.load([x, y, z], [np.zeros_like(x)] * 3, m, vf.flip3_params(*params))
        s.advance(1)
        omp_step(o, params)
        check_grid3(s.grid(), o, "one step")
        s.advance(1)
        omp_step(o, params)
        check_grid3(s.grid(), o, "two steps")
        s.advance(18)
        for _ in range(18):
            omp_step(o, params)
        pos = s.positions()
        mass = s.read("m")
    dev = np.argsort(mass.view(np.int32))
    ora = np.argsort(o.a["m"].view(np.int32))
    assert np.array_equal(mass.view(np.int32)[dev], o.a["m"].view(np.int32)[ora])
    assert np.array_equal(np.sort(mass.view(np.int32)), np.sort(m.view(np.int32)))
    for a, key in enumerate(("x", "y", "z")):
        e = o.a[key][ora]
        err = np.abs(pos[a][dev] - e)
        assert np.all(err <= 1e-4 * np.abs(e)), (key, float((err / np.abs(e)).max()))


def test_shallow_water_configuration_is_bit_exact():
    n = bench.N_SWE
    h = bench.swe_bumps()
    z = np.zeros_like(h)
    params = swe_params(9.81, 0.45, 1.0, 1.0, 1e-6)
    a = Stepper(OracleSweBackend(n, n, (0, 0, 0, 0)), n, n)
    a.set(h, z, z, params, 1e9)
    with vf.PatchSimulation(n, n) as p:
        p.load(h, z, z, params.view(np.int32))
        p.write_budget(0, 2 ** 31 - 1)
        for k in range(5):
            a.step(1)
            p.dispatch(1)
            got, want = p.read(), a.read()
            for f in range(3):
                assert np.array_equal(got[f].view(np.int32), want[f].view(np.int32)), (k, f)
            assert 2 ** 31 - 1 - p.read_budget((k + 1) % 2) == a.ticks(), k
            assert p.clamped() == a.clamped(), k


def test_batched_configuration_every_scene_matches_the_oracle():
    scenes, x, y, m = bench.batch_scenes()
    first = np.concatenate([[0], np.cumsum([c for _, c, _ in scenes])])
    table = [vf.Scene(nn, nn, c, vf.flip_params(*p)) for nn, c, p in scenes]
    xs = [x[first[k]:first[k + 1]] for k in range(len(scenes))]
    ys = [y[first[k]:first[k + 1]] for k in range(len(scenes))]
    ms = [m[first[k]:first[k + 1]] for k in range(len(scenes))]
    zs = [np.zeros_like(a) for a in xs]
    with vf.BatchSimulation(table, tait=True, sticky=bench.WALL_BATCH) as b:
        b.load(xs, ys, zs, zs, ms)
        b.advance(1)
        b.finish()
        for k, (nn, count, p) in enumerate(scenes):
            o = Flip2State(nn, nn, xs[k], ys[k], ms[k])
            o.step(np.array(vf.flip_params(*p), np.int32).view(F), (1, bench.WALL_BATCH))
            for name in ("gm", "gmu", "gmv"):
                got, want = b.read(k, name), o.g[name].astype(np.float64)
                bad = np.abs(got - want) > 1e-5 * np.maximum(1, np.abs(want))
                assert not bad.any(), (k, name, int(bad.sum()))
