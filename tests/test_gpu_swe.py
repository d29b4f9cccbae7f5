"""The shallow-water step on the GPU: bit-exact against the oracle, and the reference's ShallowWaterTest
and DiagnosticsTest run on the device through the same Stepper harness as the oracle tests.

Parity bar: bit-exact. The kernel is built without FMA contraction and with IEEE division and square
root, so every state word, speed word, budget and clamp count equals the oracle's after every step."""
import numpy as np
import pytest

import vexfluid as vf
from _oracle import F, OracleSweBackend, Stepper, slots, swe_diagnostics, swe_params, swe_ticks
from test_oracle_swe import (check_closed_box_holds_its_water, check_lake_at_rest, check_no_step_passes_the_end,
                             check_ritter_converges, check_step_follows_fastest_wave, hump)

pytestmark = pytest.mark.gpu


class GpuSweBackend:
    """PatchSimulation's raw rotation as a Stepper backend (Stepper.Gpu, Stepper.java:224-311)."""

    def __init__(self, nx, ny, edges, tile_width=0, exact=True):
        self.p = vf.PatchSimulation(nx, ny, edges)
        self.p.set_tile_width(tile_width)
        self.p.set_exact(exact)
        self.k = 0

    def load(self, h, hu, hv, params, first_speed):
        self.p.load(h, hu, hv, np.asarray(params, F).view(np.int32))

    def dispatch(self, k):
        assert k == self.p.dispatched()
        self.p.dispatch(1)

    def write_budget(self, slot, ticks):
        self.p.write_budget(slot, ticks)

    def read_budget(self, slot):
        return self.p.read_budget(slot)

    def read(self, k):
        return self.p.read()

    def clamped(self):
        return self.p.clamped()


def gpu_backend(nx, ny, edges):
    return GpuSweBackend(nx, ny, edges)


def bumps(n, seed, count=6):
    r = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:n, 0:n].astype(np.float64)
    h = np.ones((n, n))
    for _ in range(count):
        cx, cy, sig, amp = r.random() * n, r.random() * n, 2 + r.random() * n / 6, 0.1 + 0.4 * r.random()
        h += amp * np.exp(-((xx - cx) ** 2 + (yy - cy) ** 2) / (2 * sig * sig))
    return h.astype(F).ravel()


@pytest.mark.parametrize("tile_width", [0, 32, 64])
@pytest.mark.parametrize("nx,ny,edges", [(128, 96, (0, 0, 0, 0)), (130, 37, (0, 1, 1, 0)), (64, 64, (1, 1, 1, 1)),
                                         (200, 1, (0, 0, 0, 0))])
def test_steps_are_bit_exact_against_the_oracle(nx, ny, edges, tile_width):
    """Every word of state, and the clock, equal the oracle's after each of 60 steps (TMA tiles when the row
    pitch allows, plain loads otherwise; walls, open edges and a 1-D strip; the column walk over strips (0) and
    both widths of the staged tile kernel)."""
    h = bumps(max(nx, ny), 5)[: nx * ny] if ny > 1 else np.where(np.arange(nx) < nx // 2, 1.0, 0.0).astype(F)
    hu = np.zeros(nx * ny, F)
    hv = np.zeros(nx * ny, F)
    params = swe_params(9.81, 0.45, 1, 1, 1e-6)
    a = Stepper(OracleSweBackend(nx, ny, edges), nx, ny)
    b = Stepper(GpuSweBackend(nx, ny, edges, tile_width), nx, ny)
    for s in (a, b):
        s.set(h, hu, hv, params, 1e9)
    for k in range(60):
        a.step(1)
        b.step(1)
        sa, sb = a.read(), b.read()
        for f in range(3):
            assert np.array_equal(sa[f].view(np.int32), sb[f].view(np.int32)), (k, f)
        assert a.ticks() == b.ticks()
        assert a.clamped() == b.clamped()


def test_ritter_dam_break_converges_on_the_device():
    coarse, fine = check_ritter_converges(gpu_backend)
    assert abs(coarse - 0.0128) < 0.002 and abs(fine - 0.0080) < 0.002


def test_the_step_follows_the_fastest_wave_on_the_device():
    check_step_follows_fastest_wave(gpu_backend)


def test_no_step_passes_the_end_on_the_device():
    check_no_step_passes_the_end(gpu_backend)


def test_a_closed_box_holds_its_water_on_the_device():
    check_closed_box_holds_its_water(gpu_backend)


def test_a_lake_at_rest_stays_at_rest_on_the_device():
    check_lake_at_rest(gpu_backend)


def patch_advance_on_oracle(nx, ny, edges, h, hu, hv, params, grants):
    """PatchSimulation.advance (PatchSimulation.java:120-145) restated over the oracle backend."""
    from _oracle import Clock, fastest_wave
    b = OracleSweBackend(nx, ny, edges)
    b.load(h, hu, hv, params, fastest_wave(h, hu, hv, float(F(params[0])), float(F(params[4]))))
    clock, dispatched, last = Clock(), 0, 0
    out = []
    for ticks_, max_steps in grants:
        before = clock.now()
        granted = clock.grant(before + ticks_)
        b.write_budget(dispatched % 2, granted)
        left, steps = granted, 0
        while left > 0 and steps < max_steps:
            batch = min(max_steps - steps, (left + last - 1) // last) if last > 0 else 1
            for _ in range(batch):
                b.dispatch(dispatched)
                dispatched += 1
            steps += batch
            now = b.read_budget(dispatched % 2)
            if 0 < now < left:
                last = (left - now) // batch
            left = now
        clock.settle(left)
        out.append((steps, clock.now() - before, left))
    return out, b.read(dispatched)


def test_patch_simulation_advance_matches_its_restatement():
    """The runner's budget loop (batches sized from the last step, 4-byte readbacks, behind-ticks) gives
    the same Advance records and the same state as the same loop over the oracle."""
    n = 96
    h = hump(n)
    hu = np.zeros(n * n, F)
    hv = np.zeros(n * n, F)
    params = swe_params(9.81, 0.45, 1, 1, 1e-6)
    grants = [(vf.ticks(0.05), 1000), (vf.ticks(0.2), 7), (vf.ticks(0.1), 1000), (0, 10), (vf.ticks(1.0), 1000)]
    expected, state = patch_advance_on_oracle(n, n, (0, 0, 0, 0), h, hu, hv, params, grants)
    with vf.PatchSimulation(n, n) as p:
        p.load(h, hu, hv, params.view(np.int32))
        got = [p.advance(t, m) for t, m in grants]
        assert [(a.steps, a.spent_ticks, a.behind_ticks) for a in got] == expected
        assert p.now() == sum(e[1] for e in expected)
        assert p.steps() == sum(e[0] for e in expected)
        final = p.read()
        for f in range(3):
            assert np.array_equal(final[f].view(np.int32), state[f].view(np.int32))
        assert p.fastest_wave() > 0 and p.clamped() == 0


def test_device_diagnostics_match_the_host_readout():
    """Diagnostics.of (Diagnostics.java:43-81) reduced on the device, against the host restatement."""
    n = 64
    h = bumps(n, 3)
    with vf.PatchSimulation(n, n) as p:
        p.load(h, np.zeros(n * n, F), np.zeros(n * n, F), swe_params(9.81, 0.45, 1, 1, 1e-6).view(np.int32))
        p.advance(vf.ticks(0.5), 1000)
        st = p.read()
        d = p.diagnostics(9.81, float(F(1e-6)), 0.01, 1, 1)
        e = swe_diagnostics(st[0], st[1], st[2], 9.81, float(F(1e-6)), 0.01, 1, 1)
        assert abs(d[0] - e.volume) <= 1e-9 * abs(e.volume)
        for got, want in zip(d[1:6], (e.min_depth, e.max_depth, e.max_speed, e.max_froude, e.max_courant)):
            assert abs(got - want) <= 1e-12 * max(1, abs(want))
        assert d[6:] == [e.non_finite, e.negative, e.wet]


def test_every_step_kernel_gives_the_same_bits_on_a_large_grid():
    """1024 x 1024 (the learned solver's coarse grid): 20 steps with the staged tile kernel at both widths (64 the
    default) and the column walk over strips, equal to the last bit, with the same clock and fastest wave."""
    n = 1024
    h = bumps(n, 9, count=12)
    z = np.zeros(n * n, F)
    params = swe_params(9.81, 0.45, 1, 1, 1e-6).view(np.int32)
    out = []
    for width in (64, 32, 0):
        with vf.PatchSimulation(n, n) as p:
            assert p.tile_width() == 64
            p.set_tile_width(width)
            assert p.tile_width() == width
            p.load(h, z, z, params)
            a = p.advance(2 ** 31 - 1, 20)
            assert a.steps == 20
            out.append((p.read(), p.fastest_wave(), p.now()))
    for k in (1, 2):
        for f in range(3):
            assert np.array_equal(out[0][0][f].view(np.int32), out[k][0][f].view(np.int32)), (k, f)
        assert out[0][1:] == out[k][1:]
    with vf.PatchSimulation(64, 64) as p:
        with pytest.raises(vf.IllegalArgumentException):
            p.set_tile_width(48)


@pytest.mark.parametrize("nx,ny,edges", [(128, 96, (0, 0, 0, 0)), (130, 37, (0, 1, 1, 0)), (256, 200, (1, 1, 0, 0))])
def test_sixty_queued_steps_are_bit_exact_against_the_oracle(nx, ny, edges):
    """dispatch(60) queues 60 steps, each a programmatic dependent of the one before (no host wait between them):
    the state, clock and clamp count equal the oracle's after the 60 steps (TMA and plain-load tiles, walls and
    open edges)."""
    h = bumps(max(nx, ny), 7)[: nx * ny]
    z = np.zeros(nx * ny, F)
    params = swe_params(9.81, 0.45, 1, 1, 1e-6)
    a = Stepper(OracleSweBackend(nx, ny, edges), nx, ny)
    a.set(h, z, z, params, 1e9)
    a.step(60)
    with vf.PatchSimulation(nx, ny, edges) as p:
        p.load(h, z, z, params.view(np.int32))
        p.write_budget(0, 2 ** 31 - 1)
        p.dispatch(60)
        assert p.dispatched() == 60
        got = p.read()
        left = p.read_budget(0)
        assert p.clamped() == a.clamped()
    want = a.read()
    for f in range(3):
        assert np.array_equal(got[f].view(np.int32), want[f].view(np.int32)), f
    assert 2 ** 31 - 1 - left == a.ticks()


def test_overlapped_and_stream_ordered_launches_agree_to_the_bit():
    """1024 x 1024 at both tile widths: 40 steps through advance, launched as programmatic dependents and in plain
    stream order, give the same state, clock, fastest wave and clamp count."""
    n = 1024
    h = bumps(n, 11, count=12)
    z = np.zeros(n * n, F)
    params = swe_params(9.81, 0.45, 1, 1, 1e-6).view(np.int32)
    for width in (0, 32, 64):
        out = []
        for overlap in (True, False):
            with vf.PatchSimulation(n, n) as p:
                p.set_tile_width(width)
                p.set_overlap(overlap)
                p.load(h, z, z, params)
                a = p.advance(2 ** 31 - 1, 40)
                assert a.steps == 40
                out.append((p.read(), p.now(), p.fastest_wave(), p.clamped()))
        for f in range(3):
            assert np.array_equal(out[0][0][f].view(np.int32), out[1][0][f].view(np.int32)), (width, f)
        assert out[0][1:] == out[1][1:], width


# ---------------------------------------------------------------------------------- the fast mode
# Tolerance (written here): after 1 and 60 steps of smooth flow every cell's h, hu and hv within
# 2e-5 * max(1, |oracle|) of the exact arithmetic (the oracle), and the clock within one tick a step.


def fast_backend(nx, ny, edges):
    return GpuSweBackend(nx, ny, edges, exact=False)


@pytest.mark.parametrize("nx,ny,edges", [(512, 384, (0, 0, 0, 0)), (300, 130, (0, 1, 1, 0)), (130, 37, (1, 0, 0, 1)),
                                         (250, 3, (0, 0, 1, 1))])
def test_fast_mode_stays_within_its_tolerance_of_the_oracle(nx, ny, edges):
    """Both loaders of the fast mode's tile (TMA where the row pitch allows, plain loads at 130 and 250 columns),
    walls and open sides, tiles that overrun the domain on both axes."""
    h = bumps(max(nx, ny), 3, count=10)[: nx * ny]
    z = np.zeros(nx * ny, F)
    params = swe_params(9.81, 0.45, 1, 1, 1e-6)
    a = Stepper(OracleSweBackend(nx, ny, edges), nx, ny)
    b = Stepper(fast_backend(nx, ny, edges), nx, ny)
    for s in (a, b):
        s.set(h, z, z, params, 1e9)
    for steps in (1, 59):
        a.step(steps)
        b.step(steps)
        sa, sb = a.read(), b.read()
        for f in range(3):
            e = sa[f].astype(np.float64)
            err = np.abs(sb[f] - e)
            assert np.all(err <= 2e-5 * np.maximum(1, np.abs(e))), (steps, f, float(err.max()))
        assert abs(a.ticks() - b.ticks()) <= (1 if steps == 1 else 60), (a.ticks(), b.ticks())
    assert not b.b.p.exact()


def test_fast_mode_closed_box_holds_its_water():
    """ShallowWaterTest.aClosedBoxHoldsItsWater (ShallowWaterTest.java:166-195) in the fast mode: the flux form
    still moves water only between neighbours, so 300 steps keep the volume within 1e-5 and clamp nothing."""
    check_closed_box_holds_its_water(fast_backend)


def test_fast_mode_lake_at_rest_stays_at_rest():
    check_lake_at_rest(fast_backend)


def test_fast_mode_ritter_dam_break_converges():
    coarse, fine = check_ritter_converges(fast_backend)
    assert abs(coarse - 0.0128) < 0.002 and abs(fine - 0.0080) < 0.002
