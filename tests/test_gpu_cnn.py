"""The flux-correction network's device kernels against the CPU float64 restatement (oracle/cnn_ref.py).

Bars (tolerances written here):
* forward: the six face fields within 1e-2 of the largest |value| (bf16 activations; the restatement rounds at
  the same points, so what remains is fp32 summation order and an occasional one-ulp bf16 flip);
* gradient: per parameter block ||g - g_ref|| <= 2e-2 ||g_ref|| against the bf16-emulating restatement, and
  <= 8e-2 against exact float64 arithmetic; the loss within 1e-4 relative;
* the correction conserves the totals of h, hu and hv to fp32 rounding (1e-6 relative);
* training lowers the loss on a problem a network of the same shape can solve.
"""
import sys

import numpy as np
import pytest

import vexfluid as vf
from conftest import ROOT

sys.path.insert(0, str(ROOT / "oracle"))
import cnn_ref  # noqa: E402

pytestmark = pytest.mark.gpu


def smooth(rng, ny, nx, amp, k=6):
    """A smooth random field: a few random Fourier modes."""
    y, x = np.mgrid[0:ny, 0:nx].astype(np.float64)
    f = np.zeros((ny, nx))
    for _ in range(k):
        kx, ky = rng.uniform(0.05, 0.4, 2)
        f += rng.normal() * np.sin(kx * x + rng.uniform(0, 6.3)) * np.cos(ky * y + rng.uniform(0, 6.3))
    return (amp * f / k).astype(np.float32)


def random_params(rng, scale3=0.05):
    d = {}
    for name, shape in cnn_ref.SIZES:
        if name.startswith("w"):
            fan = shape[1] * shape[2]
            d[name] = rng.normal(0, np.sqrt(2.0 / fan), shape) * (scale3 if name == "w3" else 1.0)
        else:
            d[name] = rng.normal(0, 0.05, shape)
    return cnn_ref.pack(d)


def state(rng, ny, nx):
    return np.stack([1 + smooth(rng, ny, nx, 0.3), smooth(rng, ny, nx, 0.1), smooth(rng, ny, nx, 0.1)])


def blocks(g):
    d = cnn_ref.unpack(g)
    return {k: np.asarray(v, np.float64) for k, v in d.items()}


PATHS = [pytest.param(0, id="tcgen05"), pytest.param(1, id="mma_sync_rows"), pytest.param(2, id="mma_sync_row")]


@pytest.mark.parametrize("path", PATHS)
@pytest.mark.parametrize("ny,nx", [(21, 45), (40, 64), (33, 300)])
def test_forward_matches_the_restatement(ny, nx, path):
    rng = np.random.default_rng(1)
    params = random_params(rng, scale3=1.0)
    S = state(rng, ny, nx)
    with vf.FluxNet(nx, ny) as net:
        net.set_path(path)
        net.params(params)
        np.testing.assert_array_equal(net.params(), params)
        net.put(0, 0, *S)
        got = net.fluxes(0)[:, :, :6]
    want = cnn_ref.forward(S, params)["y3"]
    err = np.abs(got - want).max()
    assert err <= 1e-2 * np.abs(want).max(), (err, np.abs(want).max())


@pytest.mark.parametrize("path", PATHS)
def test_gradients_match_the_restatement(path):
    rng = np.random.default_rng(2)
    ny, nx = 24, 40
    params = random_params(rng)
    s_flux, s_res = 1e-2, 1e-3
    samples = []
    for _ in range(2):
        S = state(rng, ny, nx)
        P = S + np.stack([smooth(rng, ny, nx, 2e-3) for _ in range(3)])
        T = S + np.stack([smooth(rng, ny, nx, 2e-3) for _ in range(3)])
        samples.append((S, P.astype(np.float32), T.astype(np.float32)))
    with vf.FluxNet(nx, ny, batch=2, samples=2, s_flux=s_flux, s_res=s_res) as net:
        net.set_path(path)
        net.params(params)
        for k, (S, P, T) in enumerate(samples):
            for kind, a in enumerate((S, P, T)):
                net.put(k, kind, *a)
        g, loss = net.gradients([0, 1])
    ref_loss, ref = cnn_ref.loss_and_gradients(samples, params, s_flux, s_res)
    _, exact = cnn_ref.loss_and_gradients(samples, params, s_flux, s_res, emulate=False)
    assert abs(loss - ref_loss) <= 1e-4 * ref_loss
    got = blocks(g)
    for name in ref:
        e = np.linalg.norm(got[name] - ref[name]) / np.linalg.norm(ref[name])
        assert e <= 2e-2, (name, e)
        e64 = np.linalg.norm(got[name] - exact[name]) / np.linalg.norm(exact[name])
        assert e64 <= 8e-2, (name, e64)


def test_correction_conserves_the_totals():
    rng = np.random.default_rng(3)
    n = 64
    S = state(rng, n, n)
    params = random_params(rng, scale3=1.0)
    with vf.PatchSimulation(n, n) as sim, vf.FluxNet(n, n, s_flux=1e-3) as net:
        sim.load(S[0].ravel(), S[1].ravel(), S[2].ravel(), vf.swe_params(9.81, 0.45, 2.0, 2.0))
        net.params(params)
        before = [a.astype(np.float64).sum() for a in sim.read()]
        net.correct(sim)
        after = sim.read()
        want = cnn_ref.correct(S, params, 1e-3)
    for k in range(3):
        scale = np.abs(after[k].astype(np.float64)).sum()
        assert abs(after[k].astype(np.float64).sum() - before[k]) <= 2e-6 * scale + 1e-6
    changed = np.abs(after[0].reshape(n, n) - S[0]).max()
    assert changed > 0   # the correction did something
    assert np.abs(after[0].reshape(n, n) - want[0]).max() <= 2e-2 * changed


def test_training_lowers_the_loss():
    """Targets made by a teacher network of the same shape: P - s_flux Div G_teacher(S) = T. A student from a
    small random start must fit them."""
    rng = np.random.default_rng(4)
    n = 48
    s_flux, s_res = 1e-3, 1e-3
    teacher = random_params(rng, scale3=1.0)
    student = random_params(rng, scale3=0.01)
    nsamp = 6
    with vf.FluxNet(n, n, batch=2, samples=nsamp, s_flux=s_flux, s_res=s_res) as net:
        for k in range(nsamp):
            S = state(rng, n, n)
            P = (S + np.stack([smooth(rng, n, n, 1e-3) for _ in range(3)])).astype(np.float32)
            T = (P - s_flux * cnn_ref.divergence(cnn_ref.forward(S, teacher)["y3"])).astype(np.float32)
            for kind, a in enumerate((S, P, T)):
                net.put(k, kind, *a)
        net.params(student)
        first, plain = net.loss(list(range(nsamp))[:2])
        for it in range(300):
            net.train([(2 * it) % nsamp, (2 * it + 1) % nsamp], 2e-3)
        last, _ = net.loss(list(range(nsamp))[:2])
    assert plain > 0 and first > 0
    assert last < 0.2 * first, (first, last)
