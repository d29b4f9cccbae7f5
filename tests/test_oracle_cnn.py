"""The network's CPU restatement pinned against finite differences (float64, no bf16 rounding): the loss's
gradient with respect to every parameter block, and the correction's conservation of the totals."""
import sys

import numpy as np

from conftest import ROOT

sys.path.insert(0, str(ROOT / "oracle"))
import cnn_ref  # noqa: E402


def setup(seed=0, ny=7, nx=9):
    rng = np.random.default_rng(seed)
    d = {name: rng.normal(0, 0.3, shape) for name, shape in cnn_ref.SIZES}
    params = cnn_ref.pack(d).astype(np.float64)
    samples = []
    for _ in range(2):
        S = np.stack([1 + 0.2 * rng.random((ny, nx)), 0.1 * rng.normal(size=(ny, nx)), 0.1 * rng.normal(size=(ny, nx))])
        P = S + 1e-2 * rng.normal(size=S.shape)
        T = S + 1e-2 * rng.normal(size=S.shape)
        samples.append((S, P, T))
    return params, samples


def test_gradient_matches_finite_differences():
    params, samples = setup()
    s_flux, s_res = 0.05, 0.01
    loss, g = cnn_ref.loss_and_gradients(samples, params, s_flux, s_res, emulate=False)
    flat = np.concatenate([g[name].ravel() for name, _ in cnn_ref.SIZES])
    rng = np.random.default_rng(1)
    picks = rng.choice(len(params), 40, replace=False)
    # every block represented
    starts = np.cumsum([0] + [int(np.prod(s)) for _, s in cnn_ref.SIZES])
    picks = np.concatenate([picks, starts[:-1] + 1])
    eps = 1e-6
    for k in picks:
        p1, p2 = params.copy(), params.copy()
        p1[k] += eps
        p2[k] -= eps
        l1, _ = cnn_ref.loss_and_gradients(samples, p1, s_flux, s_res, emulate=False)
        l2, _ = cnn_ref.loss_and_gradients(samples, p2, s_flux, s_res, emulate=False)
        fd = (l1 - l2) / (2 * eps)
        assert abs(fd - flat[k]) <= 1e-5 * max(1e-3, abs(fd)) + 1e-9, (k, fd, flat[k])


def test_correction_conserves_totals_exactly_in_float64():
    params, samples = setup(2, 11, 13)
    S = samples[0][0]
    out = cnn_ref.correct(S, params.astype(np.float32), 0.01)
    for k in range(3):
        assert abs(out[k].sum() - S[k].sum()) <= 1e-12 * np.abs(S[k]).sum() + 1e-12


def test_bf16_rounding_is_to_nearest_even():
    # bf16 keeps 7 fraction bits: near 1 the spacing is 2^-7; halfway cases go to the even neighbour
    x = np.array([1.0, 1 + 2 ** -8, 1 + 2 ** -7 + 2 ** -8, 1 + 3 * 2 ** -9, 1 + 2 ** -9, -2.5])
    r = cnn_ref.bf16(x)
    assert list(r) == [1.0, 1.0, 1 + 2 ** -6, 1 + 2 ** -7, 1.0, -2.5]
