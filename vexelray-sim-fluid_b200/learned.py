"""The learned coarse shallow-water solver: the plain HLL step (ShallowWater.kernel) on a 2x-coarsened grid,
corrected once per interval by the flux-correction network (FluxNet), with a per-tile indicator whose tiles fall
back to the plain fine solver for that interval. No counterpart in the reference; its error is measured against
the plain fine solver's solution restricted to the coarse grid, and the fine solver is also its fallback.

  generate + train   fine runs (PatchSimulation at the fine resolution) give samples (S, P, T): the coarse
                     state (the fine state averaged over 2x2 cells), the plain coarse solver after one
                     interval, and the fine solver after the same interval, restricted. Both solvers advance
                     exactly the interval's ticks through the reference's tick budget (PatchSimulation.advance).
  LearnedShallowWater  coarse interval, then the correction; tiles the indicator flags are re-run on a fine
                     patch (the interval's start state copied 2x2, a margin of coarse cells around the tile,
                     open edges inside the domain) and averaged back.
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import EDGE_OPEN, EDGE_WALL, FluxNet, PatchSimulation, swe_params

G, COURANT, DRY = 9.81, 0.45, 1e-6
NEVER = 2 ** 31 - 1   # a step budget that does not stop the steps
# Coarse steps an interval may take before the learned solver gives up on it. An interval is about 16 steps of a
# still depth of 1.5; a state the correction has driven to near-dry or violent (wave speeds that shrink the step
# toward one tick) would otherwise spin here. The reference's test stepper stops a run the same way when its
# steps stop growing (vexelray-sim-fluid-core/src/test/java/dev/vexelray/sim/fluid/stencil/Stepper.java:90-93).
INTERVAL_STEP_CAP = 1024


def bumps(seed: int, n: int, count: int = 16, scale: float | None = None) -> np.ndarray:
    """h = 1 + `count` seeded Gaussian bumps on an n x n grid: amplitude U(0.1, 0.5), sigma U(20, 200) cells and
    centres uniform over a 4096-cell domain, all lengths scaled by `scale` (n / 4096 by default: on a 2048 grid,
    the 4096^2 configuration's distribution halved in sigma and centres)."""
    scale = n / 4096 if scale is None else scale
    rng = np.random.default_rng(seed)
    h = np.ones((n, n), np.float32)
    y = np.arange(n, dtype=np.float32)[:, None]
    x = np.arange(n, dtype=np.float32)[None, :]
    for _ in range(count):
        amp, sig = rng.uniform(0.1, 0.5), rng.uniform(20, 200) * scale
        cx, cy = rng.uniform(0, 4096) * scale, rng.uniform(0, 4096) * scale
        h += (amp * np.exp(-((x - cx) ** 2) / (2 * sig * sig)) * np.exp(-((y - cy) ** 2) / (2 * sig * sig))).astype(
            np.float32)
    return h


def restrict(a: np.ndarray) -> np.ndarray:
    """2x2 means (the device's restriction, on the host)."""
    ny, nx = a.shape
    return a.reshape(ny // 2, 2, nx // 2, 2).mean(axis=(1, 3), dtype=np.float64).astype(np.float32)


def fine_params(dx: float = 1.0) -> np.ndarray:
    return swe_params(G, COURANT, dx, dx, DRY)


def coarse_params(dx: float = 1.0) -> np.ndarray:
    return swe_params(G, COURANT, 2 * dx, 2 * dx, DRY)


def _empty(sim: PatchSimulation, params) -> None:
    z = np.zeros(sim.nx() * sim.ny(), np.float32)
    sim.load(z + 1, z, z, params)


class LearnedShallowWater:
    """Coarse HLL with the network's correction every `interval` ticks. `net` None: the plain coarse solver.
    `threshold` None: no fallback; else tiles of `tile` coarse cells whose relative depth jump exceeds it (at an
    interval's start) are stepped by the fine solver instead."""

    def __init__(self, nx: int, ny: int, net: FluxNet | None, interval: int, *, tile: int = 64,
                 threshold: float | None = None, margin: int = 8, dx: float = 1.0):
        self.nx, self.ny, self.net, self.interval = nx, ny, net, interval
        self.tile, self.threshold, self.margin, self.dx = tile, threshold, margin, dx
        self.coarse = PatchSimulation(nx, ny)
        self.start = PatchSimulation(nx, ny) if threshold is not None else None
        self.patches: dict = {}
        self.corrections = 0
        self.fallback_tiles = 0
        self.steps = 0

    def load(self, h, hu, hv) -> None:
        """The coarse state (nx x ny arrays)."""
        self.coarse.load(np.ravel(h), np.ravel(hu), np.ravel(hv), coarse_params(self.dx))
        if self.start is not None:
            _empty(self.start, coarse_params(self.dx))

    def load_fine(self, h, hu, hv) -> None:
        """A fine state (2ny x 2nx arrays), restricted."""
        self.load(restrict(np.asarray(h, np.float32)), restrict(np.asarray(hu, np.float32)),
                  restrict(np.asarray(hv, np.float32)))

    def read(self):
        return [a.reshape(self.ny, self.nx) for a in self.coarse.read()]

    def advance(self, total: int) -> None:
        left = int(total)
        while left > 0:
            t = min(self.interval, left)
            tripped = []
            if self.threshold is not None:
                jump = self.coarse.jump_indicator(self.tile)
                tripped = [tuple(v) for v in np.argwhere(jump > self.threshold)]
                if tripped:
                    self.start.copy_from(self.coarse)
            if self.net is not None:
                self.net.predict(self.coarse)   # from the interval's start, as the samples' S
            a = self.coarse.advance(t, INTERVAL_STEP_CAP)
            self.steps += a.steps
            if a.spent_ticks < t:
                raise RuntimeError(f"the corrected coarse state stopped advancing: {a.steps} steps covered "
                                   f"{a.spent_ticks} of the interval's {t} ticks (correction {self.corrections})")
            if self.net is not None:
                self.net.apply(self.coarse)     # to the plain interval's end, as the samples' P
                self.corrections += 1
            for ty, tx in tripped:
                self._fine_tile(int(tx), int(ty), t)
            if tripped:
                self.coarse.measure_speed()
            left -= t

    def _fine_tile(self, tx: int, ty: int, t: int) -> None:
        T, m = self.tile, self.margin
        x0, y0 = tx * T, ty * T
        w, hgt = min(T, self.nx - x0), min(T, self.ny - y0)
        bx0, by0 = max(0, x0 - m), max(0, y0 - m)
        bx1, by1 = min(self.nx, x0 + w + m), min(self.ny, y0 + hgt + m)
        edges = (EDGE_WALL if bx0 == 0 else EDGE_OPEN, EDGE_WALL if bx1 == self.nx else EDGE_OPEN,
                 EDGE_WALL if by0 == 0 else EDGE_OPEN, EDGE_WALL if by1 == self.ny else EDGE_OPEN)
        key = (bx1 - bx0, by1 - by0, edges)
        patch = self.patches.get(key)
        if patch is None:
            patch = PatchSimulation(2 * key[0], 2 * key[1], edges)
            _empty(patch, fine_params(self.dx))
            self.patches[key] = patch
        patch.prolong_from(self.start, bx0, by0)
        patch.advance(t, NEVER)
        patch.restrict_into(2 * (x0 - bx0), 2 * (y0 - by0), self.coarse, x0, y0, w, hgt)
        self.fallback_tiles += 1

    def close(self) -> None:
        for s in [self.coarse, self.start, *self.patches.values()]:
            if s is not None:
                s.close()


def trained(path=None, *, batch: int = 1, samples: int = 1):
    """The network trained for the 2048^2 configuration (learned_2048_k16.npy and its .json beside this file, made
    by train_learned.py on a B200): returns (FluxNet for the 1024^2 coarse grid, its report with interval_ticks)."""
    import json
    import pathlib
    base = pathlib.Path(path) if path else pathlib.Path(__file__).resolve().parent / "learned_2048_k16"
    report = json.loads(base.with_suffix(".json").read_text())
    net = FluxNet(report["coarse"], report["coarse"], batch=batch, samples=samples, s_flux=report["s_flux"],
                  s_res=report["s_res"])
    net.params(np.load(base.with_suffix(".npy")))
    return net, report


def coarse_step_ticks(n_fine: int, hmax: float = 1.5, dx: float = 1.0) -> int:
    """A coarse step's length in ticks at the fastest wave of a still state of depth hmax (the Courant limit the
    step itself applies, ShallowWater.java:184-192)."""
    return int(COURANT * 2 * dx / math.sqrt(G * hmax) * 1e6)


def generate_and_train(net: FluxNet, n_fine: int, seeds, *, pairs: int, spacing: int, interval: int, batch: int,
                       lr: float, steps_per_pair: float = 1, lr_end: float | None = None, seed: int = 0,
                       sample_every: int | None = None, log=None) -> dict:
    """Fine runs from the seeds (bumps), `pairs` samples each; every sample goes into the network's ring and is
    followed by `steps_per_pair` Adam steps on random batches of the ring (a fraction: one step every so many
    samples). The learning rate decays geometrically from lr to lr_end.

    Sampling: with `sample_every` the samples' start states are every `sample_every` steps of one fine run (the
    first after `sample_every` steps), and each target is a second fine solver's state an interval after a copy of
    the run's state; otherwise the run itself advances through each target, and the next start is `spacing` fine
    steps after it."""
    rng = np.random.default_rng(seed)
    nc = n_fine // 2
    fine = PatchSimulation(n_fine, n_fine)
    ahead = PatchSimulation(n_fine, n_fine) if sample_every else None
    coarse = PatchSimulation(nc, nc)
    _empty(coarse, coarse_params())
    if ahead is not None:
        _empty(ahead, fine_params())
    cap = net.samples
    filled, slot, losses = 0, 0, []
    total = int(len(seeds) * pairs * steps_per_pair)
    done, credit = 0, 0.0
    t0 = time.perf_counter()
    try:
        for s in seeds:
            h0 = bumps(s, n_fine).ravel()
            z = np.zeros_like(h0)
            fine.load(h0, z, z, fine_params())
            for _ in range(pairs):
                fine.advance(NEVER, sample_every or spacing)
                coarse.restrict_from(fine)
                net.put_state(slot, 0, coarse)
                coarse.advance(interval, NEVER)
                net.put_state(slot, 1, coarse)
                if ahead is not None:
                    ahead.copy_from(fine)
                    ahead.advance(interval, NEVER)
                    coarse.restrict_from(ahead)
                else:
                    fine.advance(interval, NEVER)
                    coarse.restrict_from(fine)
                net.put_state(slot, 2, coarse)
                filled = min(filled + 1, cap)
                slot = (slot + 1) % cap
                credit += steps_per_pair
                while credit >= 1.0:
                    credit -= 1.0
                    frac = done / max(1, total - 1)
                    rate = lr if lr_end is None else lr * (lr_end / lr) ** min(1.0, frac)
                    pick = rng.choice(filled, size=min(batch, filled), replace=False)
                    losses.append(net.train(pick, rate))
                    done += 1
            if log:
                recent = losses[-max(1, int(pairs * steps_per_pair)):]
                log(f"seed {s}: loss {np.mean(recent) if recent else float('nan'):.4g}  ({time.perf_counter() - t0:.1f} s)")
    finally:
        fine.close()
        if ahead is not None:
            ahead.close()
        coarse.close()
    return {"losses": losses, "seconds": time.perf_counter() - t0}


def _fine_run(n_fine: int, seed: int, fine_steps: int):
    """The fine solver for `fine_steps` steps from the seed's bumps: (start h, ticks spent, steps, seconds, the end
    state's h restricted)."""
    h0 = bumps(seed, n_fine)
    z = np.zeros_like(h0)
    with PatchSimulation(n_fine, n_fine) as fine:
        fine.load(h0.ravel(), z.ravel(), z.ravel(), fine_params())
        fine.advance(1, NEVER)   # one tick: warm-up of the launch path without moving the state much
        fine.load(h0.ravel(), z.ravel(), z.ravel(), fine_params())
        t0 = time.perf_counter()
        a = fine.advance(NEVER, fine_steps)
        t_fine = time.perf_counter() - t0
        ref = restrict(fine.read()[0].reshape(n_fine, n_fine))
    return h0, a.spent_ticks, a.steps, t_fine, ref


def _coarse_run(net: FluxNet | None, n_fine: int, seed: int, fine, interval: int, threshold, tile) -> dict:
    h0, span, fine_steps, t_fine, ref = fine
    z = np.zeros_like(h0)
    solver = LearnedShallowWater(n_fine // 2, n_fine // 2, net, interval, threshold=threshold, tile=tile)
    try:
        solver.load_fine(h0, z, z)
        t0 = time.perf_counter()
        solver.advance(span)
        t_coarse = time.perf_counter() - t0
        h = solver.read()[0]
    finally:
        solver.close()
    err = float(np.sqrt(np.mean((h.astype(np.float64) - ref) ** 2)))
    return {"seed": seed, "ticks": int(span), "fine_steps": int(fine_steps), "coarse_steps": solver.steps,
            "corrections": solver.corrections, "fallback_tiles": solver.fallback_tiles, "h_rms_error": err,
            "fine_s": t_fine, "coarse_s": t_coarse, "speedup": t_fine / t_coarse,
            "fine_cell_updates_per_s": n_fine * n_fine * fine_steps / t_fine,
            "equivalent_fine_cell_updates_per_s": n_fine * n_fine * fine_steps / t_coarse}


def evaluate(net: FluxNet | None, n_fine: int, seed: int, fine_steps: int, interval: int, *,
             threshold: float | None = None, tile: int = 64) -> dict:
    """One held-out run: the fine solver for `fine_steps` steps, then the coarse solver (with the network, or plain
    when net is None) over the same ticks from the restricted start; h's RMS error against the fine end state
    restricted, and both runs' times (device work and host synchronisation, from the first dispatch to the end
    state on the device)."""
    return _coarse_run(net, n_fine, seed, _fine_run(n_fine, seed, fine_steps), interval, threshold, tile)


def evaluate_pair(net: FluxNet, n_fine: int, seed: int, fine_steps: int, interval: int, *,
                  threshold: float | None = None, tile: int = 64) -> tuple[dict, dict]:
    """evaluate(None, ...) and evaluate(net, ...) against one fine run: (plain, learned)."""
    fine = _fine_run(n_fine, seed, fine_steps)
    return (_coarse_run(None, n_fine, seed, fine, interval, threshold, tile),
            _coarse_run(net, n_fine, seed, fine, interval, threshold, tile))
