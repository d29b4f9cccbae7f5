"""Surface tension on the 3D path (Tension3.java, Flip3Step with tension) on the GPU, against the oracle and the
reference's Tension3Test.

Parity bars (tolerances written here):
* the grid velocity with tension over the device's own scatter: bit-exact against the oracle's colour, blurs,
  stress and gridWithTension over the same grid (both round every operation once, in the reference's order);
* positions after 20 steps of a drop with tension: |gpu - oracle| <= 1e-4 * |oracle| per coordinate, as for the
  step without tension;
* Tension3Test's own bounds: a drop's Laplace pressure (Tension3Test.java:127-150) and a drop on the floor that
  comes to rest (Tension3Test.java:160-233).
"""
import math

import numpy as np
import pytest

import vexfluid as vf
from _oracle import F, WALL, Flip3State, JavaRandom, check_laplace, drop3, drop_pressure, flip3_params, stable_step

pytestmark = pytest.mark.gpu


def ball(nx, ny, nz, centre, radius, ppc=8, seed=0):
    """ppc particles uniform in each cell whose centre lies within radius of ``centre``, mass 1/ppc."""
    cells = np.array([(i, j, k) for k in range(nz) for j in range(ny) for i in range(nx)
                      if sum((c + 0.5 - o) ** 2 for c, o in zip((i, j, k), centre)) <= radius ** 2], np.float64)
    rng = np.random.default_rng(seed)
    at = (np.repeat(cells, ppc, axis=0) + rng.random((len(cells) * ppc, 3)) * 0.999).astype(F)
    return at[:, 0].copy(), at[:, 1].copy(), at[:, 2].copy(), np.full(len(at), F(1.0 / ppc), F)


CASES = [
    # a round drop in the middle of the box
    ((40, 40, 40), [((20, 20, 20), 8.0)], (0, 0), vf.VF_P2G_TILE),
    # drops against the floor, a side wall and a corner of a box with three different sizes, reference physics
    ((24, 20, 28), [((12, 5, 14), 5.0), ((3, 12, 8), 4.0), ((20, 16, 24), 4.5)], (0, 0), vf.VF_P2G_ATOMIC),
    # the same with Tait's pressure and two sticky nodes at every wall
    ((24, 20, 28), [((12, 5, 14), 5.0), ((3, 12, 8), 4.0)], (1, 2), vf.VF_P2G_FIXED),
]


@pytest.mark.parametrize("dims,drops,physics,schedule", CASES)
def test_the_grid_with_tension_is_bit_exact_against_the_oracle(dims, drops, physics, schedule):
    nx, ny, nz = dims
    parts = [ball(nx, ny, nz, c, r, seed=k) for k, (c, r) in enumerate(drops)]
    x, y, z, m = (np.concatenate([p[a] for p in parts]) for a in range(4))
    rng = np.random.default_rng(9)
    vel = [(rng.standard_normal(len(x)) * 2).astype(F) for _ in range(3)]
    p = (1e-3, 0.0, -30.0, 0.0, 400.0, 1.0, 80.0)
    with vf.ParticleSimulation3(nx, ny, nz, len(x), tension=True, tait=bool(physics[0]), sticky=physics[1],
                                schedule=schedule) as s:
        s.load([x, y, z], vel, m, vf.flip3_params(*p))
        s.run(vf.VF3_PASS_SORT | vf.VF3_PASS_CLEAR | vf.VF3_PASS_SCATTER)
        grid = s.grid()
        got = [s.read(k) for k in ("gu", "gv", "gw")]
    o = Flip3State(nx, ny, nz, x, y, z, m)
    for f, key in enumerate(("gm", "gmu", "gmv", "gmw")):
        o.g[key][:] = grid[f]
    o.tension_grid(flip3_params(*p), physics)
    for a, key in enumerate(("gu", "gv", "gw")):
        bad = np.flatnonzero(got[a].view(np.int32) != o.g[key].view(np.int32))
        assert bad.size == 0, (key, bad[:5], got[a][bad[:5]], o.g[key][bad[:5]])
    # the tension moved the surface: the same grid without sigma differs there
    o0 = Flip3State(nx, ny, nz, x, y, z, m)
    for f, key in enumerate(("gm", "gmu", "gmv", "gmw")):
        o0.g[key][:] = grid[f]
    o0.tension_grid(flip3_params(*p[:6], 0.0), physics)
    assert any((o0.g[k] != o.g[k]).any() for k in ("gu", "gv", "gw"))


@pytest.mark.parametrize("schedule", [vf.VF_P2G_TILE, vf.VF_P2G_ATOMIC, vf.VF_P2G_FIXED])
def test_twenty_steps_of_a_drop_follow_the_oracle(schedule):
    n = 40
    x, y, z, m, _ = drop3(n, radius=8.0)
    m = (m.view(np.int32) + np.arange(len(m), dtype=np.int32)).view(F)   # a distinct mass tags each particle
    bulk = 200.0 ** 2
    p = (stable_step(bulk, 1, 20, 0.3), 0.0, 0.0, 0.0, bulk, 1.0, 0.01 * bulk * 8)
    o = Flip3State(n, n, n, x, y, z, m)
    with vf.ParticleSimulation3(n, n, n, len(x), tension=True, schedule=schedule) as s:
        s.load([x, y, z], [np.zeros_like(x)] * 3, m, vf.flip3_params(*p))
        s.advance(20)
        pos = s.positions()
        mass = s.read("m")
    for _ in range(20):
        o.step(flip3_params(*p), tension=True)
    dev = np.argsort(mass.view(np.int32))
    ora = np.argsort(o.a["m"].view(np.int32))
    assert np.array_equal(mass.view(np.int32)[dev], o.a["m"].view(np.int32)[ora])
    for a, key in enumerate(("x", "y", "z")):
        e = o.a[key][ora]
        err = np.abs(pos[a][dev] - e)
        assert np.all(err <= 1e-4 * np.abs(e)), (key, float((err / np.abs(e)).max()))


class GpuDrop:
    """A 40^3 box with tension on the device, for drop_pressure."""

    def __init__(self, x, y, z, m, p):
        self.s = vf.ParticleSimulation3(40, 40, 40, len(x), tension=True)
        self.s.load([x, y, z], [np.zeros_like(x)] * 3, m, vf.flip3_params(*p))

    def step(self):
        self.s.advance(1)

    def read(self, name):
        return self.s.read(name)


def test_a_drops_pressure_is_twice_sigma_over_its_radius_on_the_device():
    """Tension3Test.aDropsPressureIsTwiceSigmaOverItsRadius (Tension3Test.java:127-150), its bounds."""
    sims = []

    def pressure(radius, sigma):
        def make(*a):
            sims.append(GpuDrop(*a))
            return sims[-1]
        out = drop_pressure(make, radius=radius, sigma=sigma)
        sims[-1].s.close()
        return out

    check_laplace(pressure)


def test_a_drop_on_the_floor_comes_to_rest_on_the_device():
    """Tension3Test.aDropOnTheFloorComesToRest (Tension3Test.java:160-233): a column falls and gathers into one drop
    on the floor, which must not turn over (rise up its middle) once the splash has had four seconds."""
    n, ppc = 40, 8
    g = 9.81 * (n - 1)
    fall = math.sqrt(2 * g * 30)
    bulk = 25 * fall * fall
    capillary = 10.0 * (n - 3) / 45
    dt = stable_step(bulk, 1, 2.5 * fall, 0.2)
    r = JavaRandom(1)
    count = 16 * 30 * 20 * ppc
    at = np.empty((3, count), F)
    k = 0
    for layer in range(12, 32):
        for row in range(30):
            for col in range(16):
                for s in range(ppc):
                    cell = (col, row, layer)
                    for a in range(3):
                        q = (F((s >> a) & 1) + F(0.25) + F(0.5) * r.next_float()) / F(2)
                        at[a, k] = (WALL + F(cell[a])) + q
                    k += 1
    m = np.full(count, F(1.0 / ppc), F)
    settle = math.ceil(4 / dt)
    steps = math.ceil(6 / dt)
    rise = energy = 0.0
    samples = 0
    with vf.ParticleSimulation3(n, n, n, count, tension=True) as sim:
        sim.load([at[0], at[1], at[2]], [np.zeros(count, F)] * 3, m,
                 vf.flip3_params(dt, 0, -g, 0, bulk, 1, g * capillary * capillary))
        done = 0
        for s in range(steps):
            if s < settle or s % 500 != 0:
                continue
            sim.advance(s + 1 - done)
            done = s + 1
            pos = sim.positions()
            vel = sim.velocities()
            cx, cz = pos[0].astype(np.float64).mean(), pos[2].astype(np.float64).mean()
            energy += float(0.5 * sum((v.astype(np.float64) ** 2) for v in vel).sum()) / count
            middle = np.hypot(pos[0] - cx, pos[2] - cz) < 3
            rise += float(vel[1][middle].astype(np.float64).sum()) / max(int(middle.sum()), 1)
            samples += 1
        sim.advance(steps - done)
    rise /= samples
    energy /= samples
    assert abs(rise) < 5, f"the drop turns over, rising up its middle at {rise}"
    assert energy < 120, f"the settled drop keeps kinetic energy {energy} a unit mass"
