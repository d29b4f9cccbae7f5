"""3D MLS-MPM on the GPU against the oracle and the reference's Flip3Test.

Parity bars (tolerances written here):
* grid mass and momentum after one scatter: per node |gpu - oracle| <= 1e-5 * max(1, |oracle|)
  (ScatterTest.java:140's per-node bound; node masses are O(1) in these units);
* particle positions after 100 steps: |gpu - oracle| <= 1e-4 * |oracle| per coordinate;
* the sort: cell starts and the whole permutation bit-exact against the oracle's stable counting sort;
* total mass: the particles' masses are the same multiset, bit for bit, after any number of steps.
"""
import math

import numpy as np
import pytest

import vexfluid as vf
from _oracle import F, Flip3State, JavaRandom, flip3_params, slab3, stable_step

pytestmark = pytest.mark.gpu

SCHEDULES = [("tile", vf.VF_P2G_TILE, True), ("atomic", vf.VF_P2G_ATOMIC, True), ("warp", vf.VF_P2G_WARP, True),
             ("atomic-unsorted", vf.VF_P2G_ATOMIC, False), ("fixed", vf.VF_P2G_FIXED, True), ("auto", vf.VF_P2G_AUTO, True)]


def sim3(n, count, schedule, sort, **kw):
    return vf.ParticleSimulation3(n, n, n, count, schedule=schedule, sort=sort, **kw)


@pytest.mark.parametrize("name,schedule,sort", SCHEDULES)
def test_lone_particle_falls_as_gravity_says(name, schedule, sort):
    """Flip3Test.aLoneParticleFallsAsGravitySays (Flip3Test.java:25-50)."""
    dt, g, steps = 0.01, -10.0, 5
    with sim3(12, 1, schedule, sort) as s:
        s.load([[5.3], [8.6], [6.2]], [[0], [0], [0]], [0.125], vf.flip3_params(dt, 0, g, 0, 0, 1))
        s.advance(steps)
        assert abs(s.read("v")[0] - steps * g * dt) <= 1e-5
        assert abs(s.read("y")[0] - (8.6 + g * dt * dt * steps * (steps + 1) / 2)) <= 1e-4
        assert abs(s.read("x")[0] - 5.3) <= 1e-5 and abs(s.read("z")[0] - 6.2) <= 1e-5
        assert abs(s.read("u")[0]) <= 1e-6 and abs(s.read("w")[0]) <= 1e-6
        assert abs(s.read("j")[0] - 1) <= 1e-6
        assert s.steps() == steps


def conservation_inputs(n=14, count=150):
    from test_oracle_mpm import conservation_particles3
    return conservation_particles3(n, count)


@pytest.mark.parametrize("name,schedule,sort", SCHEDULES[:3] + SCHEDULES[4:])
def test_scatter_matches_the_oracle_per_node(name, schedule, sort):
    """Flip3Test.theScatterConservesMassAndMomentum (Flip3Test.java:57-118) plus a per-node comparison: the
    device's scatter (sort, clear, scatter) against the oracle's particle-order sum."""
    n = 14
    x, y, z, m, j, vel, c = conservation_inputs(n)
    params = flip3_params(0.01, 0, -10, 0, 1e4, 1)
    fields = {"u": vel[0], "v": vel[1], "w": vel[2], "j": j}
    fields.update({f"c{a // 3}{a % 3}": c[a] for a in range(9)})
    o = Flip3State(n, n, n, x, y, z, m, **fields)
    o.clear_scatter(params)
    with sim3(n, len(x), schedule, sort) as s:
        s.load([x, y, z], [vel[0], vel[1], vel[2]], m, vf.flip3_params(0.01, 0, -10, 0, 1e4, 1))
        for k, v in fields.items():
            s.write(k, v)
        s.run(vf.VF3_PASS_SORT | vf.VF3_PASS_CLEAR | vf.VF3_PASS_SCATTER)
        grid = s.grid()
    mass = float(m.astype(np.float64).sum())
    assert abs(mass - grid[0].astype(np.float64).sum()) <= 1e-4 * mass
    for a in range(3):
        mom = float((m.astype(np.float64) * vel[a]).sum())
        assert abs(mom - grid[1 + a].astype(np.float64).sum()) <= 1e-3 * max(1, abs(mom)) + 1e-3
    for f, key in enumerate(("gm", "gmu", "gmv", "gmw")):
        e = o.g[key].astype(np.float64)
        err = np.abs(grid[f] - e)
        assert np.all(err <= 1e-5 * np.maximum(1, np.abs(e))), (name, key, float(err.max()))


def dam3(n=24, seed=71, tagged=False):
    """The Flip3Test slab (Flip3Test.java:134-166) and its step. ``tagged`` gives every particle a distinct
    mass (1/8 + k ulp(1/8), at most 0.15% above rest) so its bits identify it through any sort."""
    height, g, rho0 = 12, 200.0, 1.0
    fall = math.sqrt(2 * g * height)
    bulk = (5 * fall) ** 2 * rho0
    dt = stable_step(bulk, rho0, fall, 0.3)
    x, y, z, m = slab3(seed, n)
    if tagged:
        m = (m.view(np.int32) + np.arange(len(m), dtype=np.int32)).view(F)
    return x, y, z, m, (dt, 0.0, -g, 0.0, bulk, rho0), (height, g)


@pytest.mark.parametrize("name,schedule,sort", SCHEDULES)
def test_one_step_grid_and_hundred_step_positions_match_the_oracle(name, schedule, sort):
    n = 24
    x, y, z, m, p, _ = dam3(n, tagged=True)
    o = Flip3State(n, n, n, x, y, z, m)
    with sim3(n, len(x), schedule, sort) as s:
        s.load([x, y, z], [np.zeros_like(x)] * 3, m, vf.flip3_params(*p))
        s.advance(1)
        o.step(flip3_params(*p))
        grid = s.grid()
        for f, key in enumerate(("gm", "gmu", "gmv", "gmw")):
            e = o.g[key].astype(np.float64)
            err = np.abs(grid[f] - e)
            assert np.all(err <= 1e-5 * np.maximum(1, np.abs(e))), (name, key, float(err.max()))
        s.advance(99)
        for _ in range(99):
            o.step(flip3_params(*p))
        pos = s.positions()
        mass = s.read("m")
        # each particle is found by its mass bits, whatever order the device's sorts left it in
        dev_order = np.argsort(mass.view(np.int32))
        ora_order = np.argsort(o.a["m"].view(np.int32))
        assert np.array_equal(mass.view(np.int32)[dev_order], o.a["m"].view(np.int32)[ora_order])
        for a, key in enumerate(("x", "y", "z")):
            e = o.a[key][ora_order]
            got = pos[a][dev_order]
            err = np.abs(got - e)
            assert np.all(err <= 1e-4 * np.abs(e)), (name, key, float((err / np.abs(e)).max()))
        # total mass conserved exactly: the same masses, bit for bit
        assert np.array_equal(np.sort(mass.view(np.int32)), np.sort(m.view(np.int32)))


def test_sort_is_bit_exact_against_the_oracle():
    """The 3D sort by stencil cell: starts and permutation equal the oracle's stable counting sort."""
    n = 40
    r = np.random.default_rng(21)
    count = 20000
    x = (1 + r.random(count) * (n - 3)).astype(F)
    y = (1 + r.random(count) * (n - 3)).astype(F)
    z = (1 + r.random(count) * (n - 3)).astype(F)
    m = (0.5 + r.random(count)).astype(F)
    o = Flip3State(n, n, n, x, y, z, m)
    starts_o, keys_o, perm_o = o.sort()
    with sim3(n, count, vf.VF_P2G_TILE, True) as s:
        s.load([x, y, z], [np.zeros(count, F)] * 3, m, vf.flip3_params(1e-4, 0, 0, 0, 1, 1))
        s.run(vf.VF3_PASS_SORT)
        assert np.array_equal(s.starts(), starts_o)
        for key in ("x", "y", "z", "m"):
            assert np.array_equal(s.read(key).view(np.int32), o.a[key].view(np.int32)), key
        # a second sort of the sorted particles is the identity, from zeroed counts
        s.run(vf.VF3_PASS_SORT)
        assert np.array_equal(s.read("x").view(np.int32), o.a["x"].view(np.int32))
        assert np.array_equal(s.starts(), starts_o)


def test_sort_during_steps_keeps_the_oracle_order():
    """After steps with a sort each, the device's particle order is the oracle's (stable) order exactly:
    the G2P-fused count, the permutation and the gather agree with a from-scratch stable sort."""
    n = 24
    x, y, z, m, p, _ = dam3(n)
    with sim3(n, len(x), vf.VF_P2G_TILE, True) as s:
        s.load([x, y, z], [np.zeros_like(x)] * 3, m, vf.flip3_params(*p))
        s.advance(20)
        pos = s.positions()
        s.run(vf.VF3_PASS_SORT)
        after = s.positions()
        # the positions were already in stable sorted order of their own keys except for this
        # step's motion: re-sorting them with the oracle must give exactly the device's re-sort
        o = Flip3State(n, n, n, pos[0], pos[1], pos[2], s.read("m"))
        starts_o, _, _ = o.sort()
        for a, key in enumerate(("x", "y", "z")):
            assert np.array_equal(after[a].view(np.int32), o.a[key].view(np.int32)), key
        assert np.array_equal(s.starts(), starts_o)


@pytest.mark.parametrize("name,schedule,sort", SCHEDULES[:3])
def test_dam_break_slab_stays_water_and_does_not_move_along_z(name, schedule, sort):
    """Flip3Test.aDamBreakInASlabStaysWaterInItsBoxAndDoesNotMoveAlongZ (Flip3Test.java:134-221), the
    reference's GPU-only test, with its assertions."""
    n = 24
    x, y, z, m, p, (height, g) = dam3(n)
    dt = p[0]
    early = math.ceil(0.12 / dt)
    steps = math.ceil(0.4 / dt)
    with sim3(n, len(x), schedule, sort) as s:
        s.load([x, y, z], [np.zeros_like(x)] * 3, m, vf.flip3_params(*p))
        s.advance(early)
        moved = float(s.read("x").max()) - (1 + 6)
        s.advance(steps - early)
        px, py, pz = s.positions()
        pu, _, pw = s.velocities()
        pj = s.read("j")
    for a in (px, py, pz, pj):
        assert np.all(np.isfinite(a))
    for a in (px, py, pz):
        assert np.all((a >= 1) & (a <= n - 2))
    ritter = 2 * math.sqrt(g * height) * early * dt
    cnt = len(x)
    sj, sy = np.sort(pj), np.sort(py)
    assert 1 < moved < ritter * 1.05, (moved, ritter)
    assert sj[int(0.01 * cnt)] > 0.9 and sj[int(0.99 * cnt)] < 1.1
    assert sy[int(0.95 * cnt)] - 1 < height
    along_z = math.sqrt(np.mean(pw.astype(np.float64) ** 2)) / math.sqrt(np.mean(pu.astype(np.float64) ** 2))
    assert along_z < 0.2


def test_prepared_is_taken_once_and_closes_idempotently():
    """ParticleSimulation3.Prepared (ParticleSimulation3.java:86-102)."""
    p = vf.ParticleSimulation3.prepare(12, 12, 12, 10)
    s = vf.ParticleSimulation3(p)
    with pytest.raises(vf.IllegalStateException):
        vf.ParticleSimulation3(p)
    s.close()
    q = vf.ParticleSimulation3.prepare(12, 12, 12, 10)
    q.close()
    q.close()


def test_device_pointers_name_the_grid_and_positions():
    """ParticleSimulation3.vkBuffer (ParticleSimulation3.java:377-383) as device pointers."""
    with sim3(12, 1, vf.VF_P2G_TILE, True) as s:
        s.load([[5.3], [8.6], [6.2]], [[0], [0], [0]], [0.125], vf.flip3_params(0.01, 0, -10, 0, 0, 1))
        s.advance(1)
        s.finish()
        ptr, stride = s.device_ptr("gm")
        assert ptr and stride == 4
        ptr, stride = s.device_ptr("x")
        assert ptr and stride == 1
        with pytest.raises(vf.IllegalArgumentException):
            s.device_ptr("nope")


def test_the_exact_scatter_is_bit_exact_against_the_oracle_in_any_order():
    """VF_P2G_FIXED: the device's 64-bit fixed-point grid equals the oracle's to the bit, for the particles in two
    orders (Flip3Test's conservation particles, seed 3), and its mass is the quantized masses' sum exactly."""
    n = 14
    x, y, z, m, j, vel, c = conservation_inputs(n)
    fields = {"u": vel[0], "v": vel[1], "w": vel[2], "j": j}
    fields.update({f"c{a // 3}{a % 3}": c[a] for a in range(9)})
    params = flip3_params(0.01, 0, -10, 0, 1e4, 1)
    want = Flip3State(n, n, n, x, y, z, m, **fields).fixed_scatter(params)
    for order in (np.arange(len(x)), np.random.default_rng(4).permutation(len(x))):
        with vf.ParticleSimulation3(n, n, n, len(x), schedule=vf.VF_P2G_FIXED) as s:
            s.load([x[order], y[order], z[order]], [vel[0][order], vel[1][order], vel[2][order]], m[order],
                   vf.flip3_params(0.01, 0, -10, 0, 1e4, 1))
            s.write("j", j[order])
            for a in range(9):
                s.write(f"c{a // 3}{a % 3}", c[a][order])
            s.run(vf.VF3_PASS_SORT | vf.VF3_PASS_CLEAR | vf.VF3_PASS_SCATTER)
            got = s.fixed_grid()
        for f in range(4):
            assert np.array_equal(got[f], want[f]), f
    assert int(want[0].sum()) == int(np.rint(m.astype(np.float64) * 2.0 ** 40).astype(np.int64).sum())


def test_the_automatic_schedule_picks_by_size():
    """VF_P2G_AUTO: the warp-aggregated scatter for a scene of the reference's scale, the tile for many particles,
    for a large grid and for sparse storage; set_p2g resolves it the same way."""
    cases = [((40, 40, 40), 17408, {}, vf.VF_P2G_WARP), ((64, 64, 64), 1_600_000, {}, vf.VF_P2G_TILE),
             ((256, 256, 256), 1000, {}, vf.VF_P2G_TILE), ((40, 40, 40), 17408, {"pool_bricks": 125}, vf.VF_P2G_TILE)]
    for dims, count, kw, want in cases:
        with vf.ParticleSimulation3(*dims, count, schedule=vf.VF_P2G_AUTO, **kw) as s:
            assert s.schedule() == want, (dims, count, kw)
    with vf.ParticleSimulation3(40, 40, 40, 17408) as s:
        assert s.schedule() == vf.VF_P2G_TILE
        s.set_schedule(vf.VF_P2G_AUTO)
        assert s.schedule() == vf.VF_P2G_WARP


def test_the_nominal_mass_is_measured_at_load():
    """ParticleSimulation3's nominalMass (ParticleSimulation3.java:248-253) and compression (312-333): the smallest
    positive mass loaded, measured on the device; compression keeps the particles holding at least half of it."""
    import ctypes
    n = 24
    x, y, z, m, p, _ = dam3(n)
    m = m.copy()
    m[5] = F(0.0)                 # an empty slot: below half the nominal mass, left out
    m[9] = F(0.01)                # the smallest positive mass sets the nominal
    with vf.ParticleSimulation3(n, n, n, len(x)) as s:
        s.load([x, y, z], [np.zeros_like(x)] * 3, m, vf.flip3_params(*p))
        got = np.empty(1, F)
        vf.check(vf.lib().vf_mpm3_nominal_mass(s._h, got.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        assert got[0] == F(0.01)
        assert len(s.compression()) == len(x) - 1
        s.load([x, y, z], [np.zeros_like(x)] * 3, np.zeros_like(m), vf.flip3_params(*p))
        vf.check(vf.lib().vf_mpm3_nominal_mass(s._h, got.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        assert got[0] == np.finfo(F).max
        assert len(s.compression()) == 0


def _diag_equal(got, want):
    w = (want.min_density, want.max_density, want.low_density, want.high_density, want.mach, want.courant,
         float(want.non_finite))
    assert tuple(got) == w, (got, w)


def test_particle_diagnostics_on_the_device_match_the_oracle():
    """ParticleDiagnostics.of (ParticleDiagnostics.java:126-148) computed on the device by radix selection over
    J, against the oracle's sort of the same J read back: every field equal. Covers J after a dam-break slab's
    steps, then J rewritten with the values the reference refuses (NaN, infinities, zero, negatives), denormals,
    ties and a spread of magnitudes."""
    from _oracle import particle_diagnostics
    fall = math.sqrt(2 * 200 * 12)
    bulk = (5 * fall) ** 2
    dt = stable_step(bulk, 1.0, fall, 0.3)
    x, y, z, m = slab3(71, 24)
    with vf.ParticleSimulation3(24, 24, 24, len(x)) as s:
        s.load([x, y, z], [np.zeros_like(x)] * 3, m, vf.flip3_params(dt, 0.0, -200.0, 0.0, bulk, 1.0))
        s.advance(30)
        j = s.read("j")
        _diag_equal(s.particle_diagnostics(fall, 5 * fall, dt), particle_diagnostics(j, fall, 5 * fall, dt))
        rng = np.random.default_rng(4)
        k = np.exp(rng.normal(0, 2, len(x))).astype(F)
        k[:9] = [np.nan, np.inf, -np.inf, 0.0, -0.0, -1.0, 1e-42, 1e-40, 3e38]
        k[9:40] = np.float32(1.25)   # ties
        s.write("j", k)
        _diag_equal(s.particle_diagnostics(1.0, 2.0, 0.5), particle_diagnostics(k, 1.0, 2.0, 0.5))
        s.write("j", np.full(len(x), np.nan, F))   # nothing valid
        _diag_equal(s.particle_diagnostics(1.0, 2.0, 0.5), particle_diagnostics(np.full(len(x), np.nan, F), 1.0, 2.0, 0.5))
