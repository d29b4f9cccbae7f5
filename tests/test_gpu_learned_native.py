"""The learned coarse solver's native handle (vf_swe_learned_*) against its Python driver (learned.py), which makes
the same device calls in the same order: the coarse state after the same ticks is the same to the bit, and the
steps, corrections and fallback tiles are the same counts.

Cases: the committed network at its configuration (2048^2 fine, 1024^2 coarse); the plain coarse solver with every
tile falling back to the fine solver; the committed network's parameters on a 256^2 coarse grid with the tiles
above the median depth jump falling back, over a run that ends inside an interval; and an interval too long for
the drivers' step cap, refused by both.
"""
import pathlib

import numpy as np
import pytest

import vexfluid as vf
from vexfluid import learned as L

pytestmark = pytest.mark.gpu


def both(n_fine, net, interval, ticks, threshold, seed=11, tile=64):
    h0 = L.bumps(seed, n_fine)
    z = np.zeros_like(h0)
    py = L.LearnedShallowWater(n_fine // 2, n_fine // 2, net, interval, tile=tile, threshold=threshold)
    try:
        py.load_fine(h0, z, z)
        py.advance(ticks)
        want = [a.copy() for a in py.read()]
        want_counts = (py.steps, py.corrections, py.fallback_tiles)
    finally:
        py.close()
    with vf.LearnedSimulation(n_fine // 2, n_fine // 2, net, interval, tile=tile, threshold=threshold) as s:
        s.load(L.restrict(h0), L.restrict(z), L.restrict(z))
        s.advance(ticks)
        got = s.read()
        counts = s.counts()
    for f in range(3):
        assert np.array_equal(got[f].view(np.int32), want[f].view(np.int32)), f
    assert counts == want_counts, (counts, want_counts)
    return counts


def test_the_committed_network_at_its_configuration():
    net, report = L.trained()
    with net:
        steps, corrections, fallback = both(report["fine"], net, report["interval_ticks"],
                                            4 * report["interval_ticks"], None)
    assert corrections == 4 and fallback == 0 and steps > 0


def test_every_tile_falling_back_to_the_fine_solver():
    n = 512
    interval = 16 * L.coarse_step_ticks(n)
    steps, corrections, fallback = both(n, None, interval, 3 * interval, -1.0)
    assert corrections == 0 and fallback == 3 * 16


def test_the_tiles_above_the_median_jump_over_a_partial_interval():
    n = 512
    report_path = pathlib.Path(L.__file__).with_name("learned_2048_k16")
    import json
    report = json.loads(report_path.with_suffix(".json").read_text())
    with vf.FluxNet(n // 2, n // 2, batch=1, samples=1, s_flux=report["s_flux"], s_res=report["s_res"]) as net:
        net.params(np.load(report_path.with_suffix(".npy")))
        interval = 16 * L.coarse_step_ticks(n)
        with vf.PatchSimulation(n // 2, n // 2) as p:
            h0 = L.restrict(L.bumps(11, n))
            z = np.zeros_like(h0)
            p.load(h0.ravel(), z.ravel(), z.ravel(), L.coarse_params())
            threshold = float(np.float32(np.median(p.jump_indicator(64))))
        steps, corrections, fallback = both(n, net, interval, 3 * interval + interval // 2, threshold)
    assert corrections == 4 and 0 < fallback < 4 * 16


def test_an_interval_that_stops_advancing_is_refused_by_both_drivers():
    # An interval of about 1,600 coarse steps' ticks (100 ordinary intervals) outruns the drivers' cap of 1,024 steps
    # an interval: the state is the plain solver's, but the steps look the way they do when a correction has shrunk
    # them toward a tick, and both drivers stop instead of stepping on.
    n = 256
    interval = 100 * 16 * L.coarse_step_ticks(n)
    h0 = L.bumps(11, n)
    z = np.zeros_like(h0)
    py = L.LearnedShallowWater(n // 2, n // 2, None, interval)
    try:
        py.load_fine(h0, z, z)
        with pytest.raises(RuntimeError, match="stopped advancing"):
            py.advance(interval)
        assert py.steps == L.INTERVAL_STEP_CAP
    finally:
        py.close()
    with vf.LearnedSimulation(n // 2, n // 2, None, interval) as s:
        s.load(L.restrict(h0), L.restrict(z), L.restrict(z))
        with pytest.raises(vf.IllegalStateException, match="stopped advancing"):
            s.advance(interval)
        assert s.counts()[0] == L.INTERVAL_STEP_CAP
