"""The learned coarse shallow-water solver against the plain fine solver (its error's measure) and the plain coarse solver
(the method without the network).

* ablation: a network trained here (512^2 fine, 16 seeds) lowers the coarse solver's h RMS error on a held-out
  seed below 0.9 x the plain coarse solver's;
* the network trained for the 2048^2 configuration (committed beside the package) keeps h's RMS error <= 1e-3
  against the fine solver over 2000 fine steps on a held-out seed, and below a third of the plain coarse error;
* the per-tile fallback: tiles the indicator flags are stepped by the fine solver; with a threshold low enough to
  flag every tile the result is the fine solver's on those tiles up to the patches' margins (error below the plain
  coarse solver's);
* the correction conserves the total depth: the learned run's total h equals the start's to fp32 rounding.
"""
import numpy as np
import pytest

import vexfluid as vf
from vexfluid import learned as L

pytestmark = pytest.mark.gpu


def fresh_net(n_coarse, samples=128):
    import importlib.util
    import pathlib
    spec = importlib.util.spec_from_file_location("train_learned", pathlib.Path(L.__file__).with_name("train_learned.py"))
    t = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(t)
    net = vf.FluxNet(n_coarse, n_coarse, batch=4, samples=samples, s_flux=1e-3, s_res=1e-3)
    net.params(t.initial_params(vf))
    return net


def test_trained_network_beats_the_plain_coarse_solver():
    n, K = 512, 16
    interval = K * L.coarse_step_ticks(n)
    with fresh_net(n // 2) as net:
        L.generate_and_train(net, n, list(range(2000, 2016)), pairs=20, spacing=20, interval=interval, batch=4,
                             lr=2e-3, lr_end=2e-4, steps_per_pair=3)
        plain = L.evaluate(None, n, 7, 1000, interval)
        learned = L.evaluate(net, n, 7, 1000, interval)
    assert learned["corrections"] > 0 and plain["corrections"] == 0
    assert learned["h_rms_error"] < 0.9 * plain["h_rms_error"], (plain["h_rms_error"], learned["h_rms_error"])


def test_committed_network_meets_the_error_bar():
    net, report = L.trained()
    with net:
        plain = L.evaluate(None, report["fine"], 9, 2000, report["interval_ticks"])
        learned = L.evaluate(net, report["fine"], 9, 2000, report["interval_ticks"])
    assert learned["h_rms_error"] <= 1e-3, learned
    assert learned["h_rms_error"] < plain["h_rms_error"] / 3, (plain["h_rms_error"], learned["h_rms_error"])


def test_fallback_tiles_take_the_fine_solver():
    n, K = 512, 16
    interval = K * L.coarse_step_ticks(n)
    plain = L.evaluate(None, n, 5, 600, interval)
    everywhere = L.evaluate(None, n, 5, 600, interval, threshold=-1.0, tile=64)
    assert everywhere["fallback_tiles"] > 0
    assert everywhere["h_rms_error"] < 0.5 * plain["h_rms_error"], (plain["h_rms_error"], everywhere["h_rms_error"])
    none = L.evaluate(None, n, 5, 600, interval, threshold=1e9, tile=64)
    assert none["fallback_tiles"] == 0 and abs(none["h_rms_error"] - plain["h_rms_error"]) <= 1e-7


def test_learned_run_conserves_the_total_depth():
    net, report = L.trained()
    n = report["fine"]
    h0 = L.bumps(11, n)
    z = np.zeros_like(h0)
    s = L.LearnedShallowWater(n // 2, n // 2, net, report["interval_ticks"])
    try:
        s.load_fine(h0, z, z)
        before = s.read()[0].astype(np.float64).sum()
        s.advance(10 * report["interval_ticks"])
        after = s.read()[0].astype(np.float64).sum()
        assert s.corrections == 10
    finally:
        s.close()
        net.close()
    assert abs(after - before) <= 1e-6 * before
