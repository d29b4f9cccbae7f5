"""The learned coarse solver's host-side loop (learned.LearnedShallowWater.advance) without a GPU: the coarse patch
and the network are stand-ins that record their calls, so the interval bookkeeping and the runaway guard are
checked on the CPU.

The guard: an interval the coarse patch cannot finish within INTERVAL_STEP_CAP steps (a correction drove the state
toward dry or violent flow, and the step shrank toward a tick) raises instead of stepping on; the reference's test
stepper stops a run whose steps stop growing the same way
(vexelray-sim-fluid-core/src/test/java/dev/vexelray/sim/fluid/stencil/Stepper.java:90-93).
"""
import pytest

import vexfluid as vf
from vexfluid import learned as L


class StubPatch:
    """A coarse patch whose step covers `per_step` ticks: advance(t, cap) spends min(t, cap * per_step)."""

    def __init__(self, per_step: int):
        self.per_step = per_step
        self.calls = []

    def advance(self, ticks: int, max_steps: int) -> vf.Advance:
        self.calls.append((ticks, max_steps))
        steps = min(max_steps, -(-ticks // self.per_step))
        spent = min(ticks, steps * self.per_step)
        return vf.Advance(steps, spent, ticks - spent)


class StubNet:
    def __init__(self):
        self.calls = []

    def predict(self, coarse):
        self.calls.append("predict")

    def apply(self, coarse):
        self.calls.append("apply")


def solver(per_step: int, interval: int, net=None):
    s = object.__new__(L.LearnedShallowWater)   # the loop alone: no device patch is made
    s.nx = s.ny = 64
    s.net, s.interval, s.threshold = net, interval, None
    s.coarse, s.start, s.patches = StubPatch(per_step), None, {}
    s.corrections = s.fallback_tiles = s.steps = 0
    return s


def test_intervals_are_cut_to_the_ticks_left_and_corrected_once_each():
    net = StubNet()
    s = solver(per_step=10, interval=160, net=net)
    s.advance(400)
    assert [t for t, _ in s.coarse.calls] == [160, 160, 80]
    assert all(cap == L.INTERVAL_STEP_CAP for _, cap in s.coarse.calls)
    assert s.steps == 16 + 16 + 8 and s.corrections == 3
    assert net.calls == ["predict", "apply"] * 3


def test_an_interval_past_the_step_cap_raises_and_keeps_the_count():
    s = solver(per_step=1, interval=100 * L.INTERVAL_STEP_CAP)
    with pytest.raises(RuntimeError, match="stopped advancing"):
        s.advance(s.interval)
    assert s.steps == L.INTERVAL_STEP_CAP and s.corrections == 0


def test_an_interval_of_exactly_the_cap_completes():
    s = solver(per_step=1, interval=L.INTERVAL_STEP_CAP)
    s.advance(2 * s.interval)
    assert s.steps == 2 * L.INTERVAL_STEP_CAP
