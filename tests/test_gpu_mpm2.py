"""2D MLS-MPM and the 2D scatter schedules on the GPU, against the oracle and the reference's FlipTest,
ScatterTest, SortTest, FixedScatterTest and RelaxTest (vexelray-sim-fluid-core/src/test/java/dev/vexelray/sim/fluid/particle/).

Tolerances: per node 1e-5 * max(1, |expected|) against the f64 reference (ScatterTest.java:140); sort starts
and permutation bit-exact; fixed-point grids bit-exact."""
import math

import numpy as np
import pytest

import vexfluid as vf
from _oracle import F, Flip2State, JavaRandom, Particles, cells2, flip_column, lib as olib, fp, ip, relax_median_j
from test_oracle_mpm import (broken_runs, check_flip2_dam_break, flip2_dam_break, holds_what_the_particles_did,
                             scatter_reference)

pytestmark = pytest.mark.gpu


def test_lone_particle_falls_as_gravity_says():
    """FlipTest.aLoneParticleFallsAsGravitySays (FlipTest.java:27-47), through the Rig-style step()."""
    dt, g, steps = 0.01, -10.0, 5
    with vf.ParticleSimulation(16, 16, 1) as s:
        s.load([7.3], [12.6], [0], [0], [0.25], vf.flip_params(dt, 0, g, 0, 1))
        for _ in range(steps):
            s.step()
        assert abs(s.read("v")[0] - steps * g * dt) <= 1e-5
        assert abs(s.read("y")[0] - (12.6 + g * dt * dt * steps * (steps + 1) / 2)) <= 1e-4
        assert abs(s.read("x")[0] - 7.3) <= 1e-5
        assert abs(s.read("u")[0]) <= 1e-6
        assert abs(s.read("j")[0] - 1) <= 1e-6


def test_dam_break_stays_water_in_its_box():
    """FlipTest.aDamBreakStaysWaterInItsBox (FlipTest.java:72-127), sorted every ten steps by advance()."""
    def run(n, x, y, m, params, early, steps):
        with vf.ParticleSimulation(n, n, len(x)) as s:
            s.load(x, y, np.zeros_like(x), np.zeros_like(x), m, params.view(np.int32))
            s.advance(early, 10)
            moved = float(s.read("x").max()) - (1 + 8)
            s.advance(steps - early, 10)
            return s.read("x"), s.read("y"), s.read("j"), moved

    (x, y, j, moved), (early, steps, dt, g, height) = flip2_dam_break(run)
    check_flip2_dam_break(x, y, j, moved, early, dt, g, height)


def test_step_matches_the_oracle():
    """One step's grid per node, and 100 steps' positions per particle (sorted every 10 on both sides)."""
    n = 32
    x, y, m = flip_column(71)
    fall = math.sqrt(2 * 200 * 16)
    bulk = (5 * fall) ** 2
    dt = 0.3 / (math.sqrt(bulk) + fall)
    params = vf.flip_params(dt, 0, -200, bulk, 1)
    o = Flip2State(n, n, x, y, m)
    with vf.ParticleSimulation(n, n, len(x)) as s:
        s.load(x, y, np.zeros_like(x), np.zeros_like(x), m, params)
        s.advance(1, 10)
        o.sort()
        o.step(params.view(F))
        for key in ("gm", "gmu", "gmv"):
            e = o.g[key].astype(np.float64)
            assert np.all(np.abs(s.read(key) - e) <= 1e-5 * np.maximum(1, np.abs(e))), key
        s.advance(99, 10)
        for k in range(1, 100):
            if k % 10 == 0:
                o.sort()
            o.step(params.view(F))
        for key in ("x", "y"):
            e = o.a[key]
            got = s.read(key)
            assert np.all(np.abs(got - e) <= 1e-4 * np.abs(e)), key


@pytest.fixture(scope="module")
def jittered64():
    return Particles.jittered(63, 4, JavaRandom(7))


@pytest.mark.parametrize("mode", [vf.VF_SCATTER_GRID, vf.VF_SCATTER_PRE_REDUCED, vf.VF_SCATTER_GATHER,
                                  vf.VF_SCATTER_SEGMENTED])
def test_the_grid_holds_what_the_particles_did(jittered64, mode):
    """ScatterTest.theGridHoldsWhatTheParticlesDid (ScatterTest.java:51-64): every schedule, both orders."""
    n = 64
    for particles in (jittered64, jittered64.shuffled(JavaRandom(8))):
        given = particles.sorted_by_cell(n) if mode == vf.VF_SCATTER_GATHER else particles
        grid = vf.scatter2(mode, n, n, given.x, given.y, given.u, given.v, given.m)
        holds_what_the_particles_did(n, given, grid, label=f"mode {mode}")


def test_the_gather_is_the_same_every_run():
    """ScatterTest.theGatherIsTheSameEveryRun (ScatterTest.java:70-80)."""
    n = 64
    p = Particles.jittered(n - 1, 4, JavaRandom(9))
    a = vf.scatter2(vf.VF_SCATTER_GATHER, n, n, p.x, p.y, p.u, p.v, p.m)
    b = vf.scatter2(vf.VF_SCATTER_GATHER, n, n, p.x, p.y, p.u, p.v, p.m)
    for f in range(3):
        assert np.array_equal(a[f].view(np.int32), b[f].view(np.int32))


def test_the_gather_refuses_unsorted_particles():
    p = Particles.jittered(7, 2, JavaRandom(3)).shuffled(JavaRandom(4))
    with pytest.raises(vf.IllegalArgumentException, match="sorted by cell"):
        vf.scatter2(vf.VF_SCATTER_GATHER, 8, 8, p.x, p.y, p.u, p.v, p.m)


def test_the_segmented_sum_keeps_broken_runs_apart():
    """ScatterTest.theSegmentedSumKeepsBrokenRunsApart (ScatterTest.java:88-108)."""
    p = broken_runs()
    grid = vf.scatter2(vf.VF_SCATTER_SEGMENTED, 8, 8, p.x, p.y, p.u, p.v, p.m)
    holds_what_the_particles_did(8, p, grid, label="broken runs")


def test_a_particle_on_a_node_weighs_only_on_it():
    """ScatterTest.aParticleOnANodeWeighsOnlyOnIt (ScatterTest.java:150-164)."""
    n = 8
    gm = vf.scatter2(vf.VF_SCATTER_GRID, n, n, [3, 7, -2], [5, 7, 1e9], [1, 1, 1], [0, 0, 0], [2, 3, 5])[0]
    expected = np.zeros(n * n, F)
    expected[5 * n + 3], expected[7 * n + 7], expected[7 * n] = 2, 3, 5
    assert np.array_equal(gm, expected)


def test_a_uniform_flow_reads_back_as_itself():
    """ScatterTest.aUniformFlowReadsBackAsItself (ScatterTest.java:171-195)."""
    n = 32
    allp = Particles.jittered(n - 1, 4, JavaRandom(11))
    west = allp.where(allp.x < n / 2 - 2)
    west.u[:] = 1.25
    west.v[:] = -0.5
    gm, gmu, gmv = vf.scatter2(vf.VF_SCATTER_GRID, n, n, west.x, west.y, west.u, west.v, west.m)
    east = np.arange(n * n) % n >= n // 2
    assert np.all(gm[east] == 0) and np.all(gmu[east] == 0) and np.all(gmv[east] == 0)
    wet = (~east) & (gm > 0)
    assert np.all(np.abs(gmu[wet] / gm[wet] - 1.25) <= 1e-5) and np.all(np.abs(gmv[wet] / gm[wet] + 0.5) <= 1e-5)


def oracle_sort(p: Particles, n):
    keys = cells2(p.x, p.y, n, n)
    starts = np.zeros((n - 1) ** 2 + 1, np.int32)
    perm = np.zeros(p.count(), np.int32)
    olib().or_counting_sort(ip(keys), p.count(), (n - 1) ** 2, ip(starts), ip(perm))
    return perm, starts


def test_the_device_sorts_by_cell_bit_exactly():
    """SortTest.theDeviceSortsByCell (SortTest.java:51-61), 259^2 cells, random order: starts exactly the host's,
    and (stronger than the reference asks) the whole permutation equal to the stable order."""
    n = 260
    p = Particles.jittered(n - 1, 1, JavaRandom(21)).shuffled(JavaRandom(22))
    perm, starts = vf.sort2(n, n, p.x, p.y)
    perm_o, starts_o = oracle_sort(p, n)
    assert np.array_equal(starts, starts_o)
    assert np.array_equal(perm, perm_o)


def test_a_second_sort_starts_from_zero_counts():
    """SortTest.aSecondSortStartsFromZeroCounts (SortTest.java:68-81), through the simulation's own buffers."""
    n = 40
    first = Particles.jittered(n - 1, 3, JavaRandom(31)).shuffled(JavaRandom(32))
    second = Particles.jittered(n - 1, 3, JavaRandom(33)).shuffled(JavaRandom(34))
    with vf.ParticleSimulation(n, n, first.count()) as s:
        for p in (first, second):
            s.load(p.x, p.y, p.u, p.v, p.m, vf.flip_params(1e-4, 0, 0, 0, 1))
            s.sort()
            perm_o, starts_o = oracle_sort(p, n)
            assert np.array_equal(s.starts(), starts_o)
            assert np.array_equal(s.read("x").view(np.int32), p.x[perm_o].view(np.int32))
            assert np.array_equal(s.read("m").view(np.int32), p.m[perm_o].view(np.int32))


def test_fixed_scatter_is_bit_exact_against_the_oracle(jittered64):
    """FixedScatter (FixedScatter.java:24-60): the device's integer grid equals the host's, in any order."""
    n = 64
    for q in (jittered64, jittered64.shuffled(JavaRandom(8))):
        g = vf.fixed_scatter2(n, n, q.x, q.y, q.u, q.v, q.m, 14, 10)
        e = [np.zeros(n * n, np.int32) for _ in range(3)]
        olib().or_fixed_scatter2(n, n, fp(q.x), fp(q.y), fp(q.u), fp(q.v), fp(q.m), q.count(), 14, 10, ip(e[0]),
                                 ip(e[1]), ip(e[2]))
        for f in range(3):
            assert np.array_equal(g[f], e[f])


def c0_dam_break(seed=0):
    """The 2D configuration: 128^2 nodes (dx = 1/128), 4 particles per cell jittered in every cell whose centre lies
    in [0.05,0.55] x [0.05,0.30] (2048 cells: 8192 particles), still, m = 1/4 (rho0 = 1 per cell)."""
    n = 128
    rng = np.random.default_rng(seed)
    cx = np.arange(math.ceil(0.05 * n - 0.5), math.ceil(0.55 * n - 0.5), dtype=np.float32)
    cy = np.arange(math.ceil(0.05 * n - 0.5), math.ceil(0.30 * n - 0.5), dtype=np.float32)
    gy, gx = np.meshgrid(cy, cx, indexing="ij")
    cells = np.repeat(np.stack([gx.ravel(), gy.ravel()], 1), 4, axis=0)
    pos = (cells + rng.random(cells.shape, dtype=np.float32) * np.float32(0.999)).astype(np.float32)
    return n, np.ascontiguousarray(pos[:, 0]), np.ascontiguousarray(pos[:, 1]), np.full(len(pos), 0.25, np.float32)


def test_the_2d_configuration_matches_the_oracle():
    """Config 0: Tait k = 50 (50 n^2 in node units), rho0 = 1, g = -9.8 (n nodes/s^2), dt = 1e-4, sticky walls 3
    cells thick; sorted every 10 steps on both sides. One step's grid per node (1e-5), 100 steps' positions (1e-4),
    masses unchanged."""
    n, x, y, m = c0_dam_break()
    assert len(x) == 8192
    params = vf.flip_params(1e-4, 0, -9.8 * n, 50.0 * n * n, 1.0)
    o = Flip2State(n, n, x, y, m)
    with vf.ParticleSimulation(n, n, len(x), tait=True, sticky=3) as s:
        s.load(x, y, np.zeros_like(x), np.zeros_like(x), m, params)
        s.advance(1, 10)
        o.sort()
        o.step(params.view(F), (1, 3))
        for key in ("gm", "gmu", "gmv"):
            e = o.g[key].astype(np.float64)
            assert np.all(np.abs(s.read(key) - e) <= 1e-5 * np.maximum(1, np.abs(e))), key
        s.advance(99, 10)
        for k in range(1, 100):
            if k % 10 == 0:
                o.sort()
            o.step(params.view(F), (1, 3))
        for key in ("x", "y"):
            e = o.a[key]
            got = s.read(key)
            assert np.all(np.abs(got - e) <= 1e-4 * np.abs(e)), key
        assert np.array_equal(s.read("m"), o.a["m"])


def test_relaxation_draws_j_to_the_volume_the_mass_gives_on_the_device():
    """RelaxTest.jIsDrawnToTheVolumeTheMassGivesAndOnlyIfAskedTo (RelaxTest.java:67-80) with its bounds: J started
    at 0.9 in a box full wall to wall stays within 0.05 of 0.9 at rate 0 and is drawn into (0.97, 1.03) at rate 8."""
    def run(x, y, m, j, params, steps):
        with vf.ParticleSimulation(48, 48, len(x), relax=True) as s:
            s.load(x, y, np.zeros_like(x), np.zeros_like(x), m, params.view(np.int32))
            s.write("j", j)
            s.advance(steps, 10)
            return s.read("j")

    without = relax_median_j(run, 0.0)
    relaxed = relax_median_j(run, 8.0)
    assert abs(without - 0.9) <= 0.05, f"J moved by itself to {without}"
    assert 0.97 < relaxed < 1.03, f"relaxed J is {relaxed}, not 1"


def test_relaxing_steps_match_the_oracle():
    """A falling column with J started at 0.9 and relaxation at rate 8: one step's J per particle within 1e-5, and
    100 steps' positions and J within 1e-4 relative of the oracle's relaxing step (sorted every 10 on both sides)."""
    n = 32
    x, y, m = flip_column(71)
    fall = math.sqrt(2 * 200 * 16)
    bulk = (5 * fall) ** 2
    dt = 0.3 / (math.sqrt(bulk) + fall)
    params = vf.flip_params(dt, 0, -200, bulk, 1, relax=8.0)
    j0 = np.full(len(x), F(0.9), F)
    o = Flip2State(n, n, x, y, m, j=j0)
    with vf.ParticleSimulation(n, n, len(x), relax=True) as s:
        s.load(x, y, np.zeros_like(x), np.zeros_like(x), m, params)
        s.write("j", j0)
        s.advance(1, 10)
        o.sort()
        o.step(params.view(F), relax=True)
        assert np.all(np.abs(s.read("j") - o.a["j"]) <= 1e-5)
        assert np.any(s.read("j") != j0)
        s.advance(99, 10)
        for k in range(1, 100):
            if k % 10 == 0:
                o.sort()
            o.step(params.view(F), relax=True)
        for key in ("x", "y", "j"):
            e = o.a[key]
            got = s.read(key)
            assert np.all(np.abs(got - e) <= 1e-4 * np.abs(e)), key


def test_replayed_steps_match_the_oracle():
    """advance() from captured graphs (a sort and the ten steps after it per graph): 1, 25 and 74 steps (blocks
    and loose steps) of the falling column, positions within the 100-step bar of the oracle's sorted run."""
    n = 32
    x, y, m = flip_column(71)
    fall = math.sqrt(2 * 200 * 16)
    bulk = (5 * fall) ** 2
    dt = 0.3 / (math.sqrt(bulk) + fall)
    params = vf.flip_params(dt, 0, -200, bulk, 1)
    o = Flip2State(n, n, x, y, m)
    with vf.ParticleSimulation(n, n, len(x)) as s:
        s.set_graph(True)
        s.load(x, y, np.zeros_like(x), np.zeros_like(x), m, params)
        for count in (1, 25, 74):
            s.advance(count, 10)
        assert s.steps() == 100
        for k in range(100):
            if k % 10 == 0:
                o.sort()
            o.step(params.view(F))
        for key in ("x", "y"):
            e = o.a[key]
            got = s.read(key)
            assert np.all(np.abs(got - e) <= 1e-4 * np.abs(e)), key
