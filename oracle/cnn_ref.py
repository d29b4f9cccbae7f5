"""cnn_ref.py -- CPU float64 restatement of the flux-correction network, its loss and its gradients.

Test infrastructure only: the gradient check (tests/) compares the device's forward, loss and backward
kernels against these functions. Nothing in the product imports it.

The network has no counterpart in the reference (sibarum/vexelray-sim-fluid); it corrects the coarse
shallow-water step, whose flux form it keeps (ShallowWater.java:206-235: U' = U - rx (Fe - Fw) - ry (Fn - Fs)),
so its correction is a divergence of face fields with the walls' faces at zero.

The device rounds to bf16 at fixed points (features, weights, hidden activations, the output gradient and the
hidden gradients) and accumulates in fp32; `emulate=True` rounds at the same points, so the remaining
difference is the fp32 summation order.
"""
import numpy as np

TAPS, HID, FEAT, FLUX = 25, 32, 3, 6
SCALE_H, SCALE_Q = 4.0, 4.0
SIZES = [("w1", (HID, TAPS, FEAT)), ("b1", (HID,)), ("w2", (HID, TAPS, HID)), ("b2", (HID,)),
         ("w3", (FLUX, TAPS, HID)), ("b3", (FLUX,))]
COUNT = sum(int(np.prod(s)) for _, s in SIZES)


def bf16(x):
    """Round to the nearest bf16 (ties to even), as float64."""
    f = np.asarray(x, np.float64).astype(np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params):
    out, at = {}, 0
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = np.asarray(params[at:at + n], np.float64).reshape(shape)
        at += n
    return out


def pack(d):
    return np.concatenate([d[name].ravel() for name, _ in SIZES]).astype(np.float32)


def conv5(x, w, b=None):
    """5x5 convolution with zero padding: x (H, W, Cin), w (Cout, 25, Cin) -> (H, W, Cout)."""
    H, W, _ = x.shape
    xp = np.pad(x, ((2, 2), (2, 2), (0, 0)))
    out = np.zeros((H, W, w.shape[0]))
    for t in range(TAPS):
        ky, kx = divmod(t, 5)
        out += xp[ky:ky + H, kx:kx + W, :] @ w[:, t, :].T
    return out if b is None else out + b


def conv5_transpose(dy, w):
    """The input gradient of conv5: dx[q, ci] = sum over taps and co of w[co, tap, ci] dy[q - (ky-2, kx-2), co]."""
    H, W, _ = dy.shape
    dyp = np.pad(dy, ((2, 2), (2, 2), (0, 0)))
    out = np.zeros((H, W, w.shape[2]))
    for t in range(TAPS):
        ky, kx = divmod(t, 5)
        out += dyp[4 - ky:4 - ky + H, 4 - kx:4 - kx + W, :] @ w[:, t, :]
    return out


def conv5_wgrad(x, dy):
    """dW[co, tap, ci] = sum over pixels of dy[p, co] x[p + (ky-2, kx-2), ci]."""
    H, W, C = x.shape
    xp = np.pad(x, ((2, 2), (2, 2), (0, 0)))
    dw = np.zeros((dy.shape[2], TAPS, C))
    for t in range(TAPS):
        ky, kx = divmod(t, 5)
        dw[:, t, :] = dy.reshape(-1, dy.shape[2]).T @ xp[ky:ky + H, kx:kx + W, :].reshape(-1, C)
    return dw


def features(state):
    h, hu, hv = (np.asarray(a, np.float64) for a in state)
    return np.stack([(h - 1.0) * SCALE_H, hu * SCALE_Q, hv * SCALE_Q], axis=-1)


def forward(state, params, emulate=True):
    r = bf16 if emulate else (lambda a: np.asarray(a, np.float64))
    p = unpack(params)
    x0 = r(features(state))
    a1 = r(np.maximum(conv5(x0, r(p["w1"]), p["b1"]), 0))
    a2 = r(np.maximum(conv5(a1, r(p["w2"]), p["b2"]), 0))
    y3 = conv5(a2, r(p["w3"]), p["b3"])
    return {"x0": x0, "a1": a1, "a2": a2, "y3": y3, "p": p}


def divergence(y3):
    """Per component c (h, hu, hv): G_e(i,j) - G_e(i-1,j) + G_n(i,j) - G_n(i,j-1), walls' faces zero.
    y3 (H, W, 6): east faces in channels 0-2, north faces in 3-5. Returns (3, H, W)."""
    H, W, _ = y3.shape
    ge = y3[:, :, 0:3].copy()
    gn = y3[:, :, 3:6].copy()
    ge[:, W - 1, :] = 0
    gn[H - 1, :, :] = 0
    d = ge.copy()
    d[:, 1:, :] -= ge[:, :-1, :]
    d += gn
    d[1:, :, :] -= gn[:-1, :, :]
    return np.moveaxis(d, -1, 0)


def correct(state, params, s_flux):
    """The corrected state: U - s_flux Div G, depth kept >= 0."""
    y3 = forward(state, params)["y3"]
    out = np.asarray(state, np.float64) - s_flux * divergence(y3)
    out[0] = np.maximum(out[0], 0)
    return out


def loss_and_gradients(samples, params, s_flux, s_res, emulate=True):
    """samples: list of (S, P, T), each (3, H, W). Returns (loss, gradient as the packed parameter vector)."""
    r = bf16 if emulate else (lambda a: np.asarray(a, np.float64))
    grads = {name: np.zeros(shape) for name, shape in SIZES}
    total, terms = 0.0, 0
    for S, P, T in samples:
        f = forward(S, params, emulate)
        p = f["p"]
        res = np.asarray(P, np.float64) - s_flux * divergence(f["y3"]) - np.asarray(T, np.float64)
        total += float(np.sum((res / s_res) ** 2))
        terms += res.size
        # d(sum (res/s_res)^2 / 2)/d y3 (the device stores it in bf16 before dividing by the number of terms)
        k = s_flux / (s_res * s_res)
        H, W = res.shape[1:]
        dy3 = np.zeros((H, W, 6))
        rr = np.moveaxis(res, 0, -1)
        dy3[:, :W - 1, 0:3] = k * (rr[:, 1:, :] - rr[:, :-1, :])
        dy3[:H - 1, :, 3:6] = k * (rr[1:, :, :] - rr[:-1, :, :])
        dy3 = r(dy3)
        grads["w3"] += conv5_wgrad(f["a2"], dy3)
        grads["b3"] += dy3.sum(axis=(0, 1))
        dy2 = r(conv5_transpose(dy3, r(p["w3"])) * (f["a2"] > 0))
        grads["w2"] += conv5_wgrad(f["a1"], dy2)
        grads["b2"] += dy2.sum(axis=(0, 1))
        dy1 = r(conv5_transpose(dy2, r(p["w2"])) * (f["a1"] > 0))
        grads["w1"] += conv5_wgrad(f["x0"], dy1)
        grads["b1"] += dy1.sum(axis=(0, 1))
    loss = total / (2.0 * terms)
    return loss, {k: v / terms for k, v in grads.items()}
