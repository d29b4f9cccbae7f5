#!/usr/bin/env python
"""bench.py -- the 3D MLS-MPM dam break at 256^3 (8,156,736 particles), one B200 per rank.

A step is one full ParticleSimulation3.advance(1): the per-step counting sort by stencil cell, the
scatter (P2G), the grid update and the gather (G2P), on inputs resident in HBM. The last stdout line
is the headline: particle-steps/s for the whole job, the P2G+G2P roofline against the measured HBM
bandwidth, the same metric end to end through the public API (host arrays in, positions out), the
oracle's threaded CPU step as the CPU baseline, and the SM clocks sampled in the timed region.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--only swe,batch,...]

--only runs sub-measurements of the other configurations (shallow water, the 2D dam break, the literal
box, the batched scenes, the learned solver, the P2G schedules, tension and sparse storage) first, each
printed as one JSON line ahead of the headline.

Under torchrun each rank runs an independent replica on its own GPU (the 3D step does not shard
across GPUs here: replicas only); the time is the max over ranks and the value the sum of work.
"""
from __future__ import annotations

import argparse
import ctypes
import importlib.util
import json
import math
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
PKG = ROOT / "vexelray-sim-fluid_b200"

# ---------------------------------------------------------------------------------------------- workload

N3 = 256                    # grid nodes per axis, dx = 1/256
PPC3 = 8                    # particles per cell
BOX3 = ((0.05, 0.45), (0.05, 0.4325), (0.05, 0.45))   # 8.16M particles at 8 ppc (the config's "~8.2M")
BOX3_LITERAL = ((0.05, 0.45), (0.05, 0.65), (0.05, 0.45))   # the literal box: 12,734,496 particles
DT3 = 5e-5
G_SI = 9.8
SEED3 = 1
WORKLOAD3 = ("3D MLS-MPM APIC dam break, 256^3 nodes, dx=1/256, 8 ppc jittered (seed 1) in "
             "[0.05,0.45]x[0.05,0.4325]x[0.05,0.45] = 8,156,736 particles, dt=5e-5, g=-9.8 m/s^2, "
             "counting sort by stencil cell every step")

N_SWE = 4096
SEED_SWE = 2


def package():
    if "vexfluid" in sys.modules:
        return sys.modules["vexfluid"]
    spec = importlib.util.spec_from_file_location("vexfluid", PKG / "__init__.py", submodule_search_locations=[str(PKG)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["vexfluid"] = mod
    spec.loader.exec_module(mod)
    return mod


def dam3(box=BOX3):
    """Seeded particles of the 3D config: every cell whose centre lies in the box, PPC3 jittered particles
    each (cell + U*0.999 per axis, as the reference's tests fill cells), z-major order."""
    n = N3
    rng = np.random.default_rng(SEED3)
    ranges = []
    for lo, hi in box:
        a, b = lo * n, hi * n
        c0 = math.ceil(a - 0.5)
        c1 = math.ceil(b - 0.5)
        ranges.append(np.arange(c0, c1, dtype=np.float32))
    cz, cy, cx = np.meshgrid(ranges[2], ranges[1], ranges[0], indexing="ij")
    cells = np.stack([cx.ravel(), cy.ravel(), cz.ravel()], axis=1)
    cells = np.repeat(cells, PPC3, axis=0)
    jitter = (rng.random(cells.shape, dtype=np.float32) * np.float32(0.999)).astype(np.float32)
    pos = (cells + jitter).astype(np.float32)
    x, y, z = (np.ascontiguousarray(pos[:, a]) for a in range(3))
    m = np.full(len(x), np.float32(1.0 / PPC3), np.float32)
    g = -G_SI * n
    height = len(ranges[1])
    fall = math.sqrt(2 * -g * height)
    bulk = (5 * fall) ** 2
    return x, y, z, m, (DT3, 0.0, g, 0.0, bulk, 1.0)


def swe_bumps(n=N_SWE):
    """The shallow-water config: h = 1 + 16 seeded Gaussian bumps (amplitude U(0.1,0.5), sigma U(20,200)
    cells, centres uniform), hu = hv = 0."""
    rng = np.random.default_rng(SEED_SWE)
    h = np.ones((n, n), np.float32)
    y = np.arange(n, dtype=np.float32)[:, None]
    x = np.arange(n, dtype=np.float32)[None, :]
    for _ in range(16):
        amp, sig = rng.uniform(0.1, 0.5), rng.uniform(20, 200)
        cx, cy = rng.uniform(0, n), rng.uniform(0, n)
        h += (amp * np.exp(-((x - cx) ** 2) / (2 * sig * sig)) * np.exp(-((y - cy) ** 2) / (2 * sig * sig))).astype(np.float32)
    return h.ravel()


N_BATCH = 256
SEED_BATCH = 3
BATCH_GRIDS = (64, 128, 256, 512)
BATCH_NP = (4096, 262144)
K_TAIT = 50.0               # Tait k in m^2/s^2 (rho0 = 1); in node units k n^2
WALL_BATCH = 3              # sticky wall thickness in nodes


def dam2_scene(rng, n, count, ppc=4):
    """One dam-break scene of the 2D config's physics on an n x n grid (dx = 1/n): `count` particles filling a
    box at the lower-left corner, `ppc` per cell where the box fits (more where it cannot), its aspect
    ratio drawn from rng; each cell's particles jittered (cell + U*0.999). Returns x, y, m, Flip.params values:
    g = -9.8 n node/s^2, Tait k = 50 n^2, rho0 = 1, dt = 1e-4 capped at a Courant number of 0.4 of the Tait
    sound speed sqrt(7k) (so the 512^2 scenes step 4.2e-5)."""
    area = count / ppc
    aspect = math.exp(rng.uniform(math.log(0.5), math.log(2.0)))
    lo = WALL_BATCH + 1
    span = n - 2 * lo
    w = int(min(span, max(1, round(math.sqrt(area * aspect)))))
    h = int(min(span, max(1, math.ceil(area / w))))
    cells = w * h
    k = np.arange(count)
    cell = k % cells
    cx = (lo + cell % w).astype(np.float32)
    cy = (lo + cell // w).astype(np.float32)
    j = rng.random((2, count), dtype=np.float32) * np.float32(0.999)
    x = (cx + j[0]).astype(np.float32)
    y = (cy + j[1]).astype(np.float32)
    m = np.full(count, np.float32(cells / count), np.float32)
    bulk = K_TAIT * n * n
    dt = min(1e-4, 0.4 / (math.sqrt(7 * K_TAIT) * n))
    return x, y, m, (dt, 0.0, -G_SI * n, bulk, 1.0)


def batch_scenes(seed=SEED_BATCH, count=N_BATCH, np_range=BATCH_NP, grids=BATCH_GRIDS):
    """The batched config: `count` dam-break scenes, grids uniform over `grids`, particle counts log-uniform in
    np_range, box aspect from the seed. Returns (scenes as (n, particles, params)), x, y, m concatenated."""
    rng = np.random.default_rng(seed)
    scenes, xs, ys, ms = [], [], [], []
    for _ in range(count):
        n = int(rng.choice(grids))
        npart = int(round(math.exp(rng.uniform(math.log(np_range[0]), math.log(np_range[1])))))
        x, y, m, params = dam2_scene(rng, n, npart)
        scenes.append((n, npart, params))
        xs.append(x)
        ys.append(y)
        ms.append(m)
    return scenes, np.concatenate(xs), np.concatenate(ys), np.concatenate(ms)


# ---------------------------------------------------------------------------------------------- helpers

class Clocks:
    """SM clock and throttle reasons sampled during a timed region: NVML polled every 2 ms from a thread (the timed
    region of the default run is tens of milliseconds), or nvidia-smi every 200 ms where NVML cannot be loaded."""

    REASONS = {"hw_slowdown": 0x2, "sw_power_cap": 0x4, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20}
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.samples: list[tuple[float, int]] = []   # (SM MHz, reason bits)
        self.max_mhz = None
        self.proc = None
        self.stop = threading.Event()
        self.thread = None
        self.nvml = None

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            handle = pynvml.nvmlDeviceGetHandleByIndex(self.device)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(handle, pynvml.NVML_CLOCK_SM))
            self.nvml = pynvml

            def poll():
                while not self.stop.is_set():
                    mhz = pynvml.nvmlDeviceGetClockInfo(handle, pynvml.NVML_CLOCK_SM)
                    bits = pynvml.nvmlDeviceGetCurrentClocksEventReasons(handle)
                    self.samples.append((float(mhz), int(bits)))
                    time.sleep(0.002)

            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            time.sleep(0.005)
        except Exception:
            self.nvml = None
            try:
                self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                              "--format=csv,noheader,nounits", "-lms", "200"],
                                             stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self.thread = threading.Thread(target=self._read_smi, daemon=True)
                self.thread.start()
            except OSError:
                self.proc = None
        return self

    def _read_smi(self):
        for line in self.proc.stdout:
            f = [v.strip() for v in line.split(",")]
            if len(f) < 9:
                continue
            try:
                mhz, self.max_mhz = float(f[1]), float(f[2])
            except ValueError:
                continue
            bits = 0
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), f[5:9]):
                if v.lower().startswith("active"):
                    bits |= self.REASONS[name]
            self.samples.append((mhz, bits))

    def __exit__(self, *exc):
        self.stop.set()
        if self.nvml is not None:
            self.thread.join(timeout=1)
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"], "samples": 0}
        reasons = sorted({name for name, bit in self.REASONS.items() for _, b in self.samples if b & bit})
        return {"sm_mhz": statistics.median(s for s, _ in self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.samples),
                "source": "nvml every 2 ms" if self.nvml is not None else "nvidia-smi every 200 ms"}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measured_tensor_peak():
    """Dense bf16 TFLOP/s: the burst figure (a kernel timed alone) and its kind."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["bf16_tflops"]), "measured"
    return 1590.0, "fallback"


def profiled_traffic(kernel: str):
    """dram bytes per launch of a kernel from the committed ncu summary, scaled to this workload, or None."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    e = d.get(kernel)
    return None if e is None else e.get("bytes_per_launch_full")


class Dist:
    """torch.distributed plumbing for N ranks (gloo: only a barrier and a max of device times cross ranks)."""

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
            self.dist = dist

    def barrier(self):
        if self.world > 1:
            self.dist.barrier()

    def max(self, v: float) -> float:
        if self.world == 1:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v: float) -> float:
        if self.world == 1:
            return v
        import torch
        t = torch.tensor([v], dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.dist.destroy_process_group()


# ---------------------------------------------------------------------------------------------- CPU side

def c0_dam_break(seed=0):
    """The 2D configuration: 128^2 nodes (dx = 1/128), 4 particles per cell jittered in every cell whose centre lies
    in [0.05,0.55] x [0.05,0.30] (2048 cells: 8192 particles), still, m = 1/4; Tait k = 50 (50 n^2 in node
    units), rho0 = 1, g = -9.8 m/s^2 (n nodes/s^2), dt = 1e-4, sticky walls 3 cells thick."""
    n = 128
    rng = np.random.default_rng(seed)
    cx = np.arange(math.ceil(0.05 * n - 0.5), math.ceil(0.55 * n - 0.5), dtype=np.float32)
    cy = np.arange(math.ceil(0.05 * n - 0.5), math.ceil(0.30 * n - 0.5), dtype=np.float32)
    gy, gx = np.meshgrid(cy, cx, indexing="ij")
    cells = np.repeat(np.stack([gx.ravel(), gy.ravel()], 1), 4, axis=0)
    pos = (cells + rng.random(cells.shape, dtype=np.float32) * np.float32(0.999)).astype(np.float32)
    x, y = np.ascontiguousarray(pos[:, 0]), np.ascontiguousarray(pos[:, 1])
    return n, x, y, np.full(len(x), 0.25, np.float32), (1e-4, 0.0, -G_SI * n, K_TAIT * n * n, 1.0)


def run_c0(args, vf, dist):
    """The 2D configuration on the GPU (sorted every 10 steps, one scene per launch sequence) and the oracle's
    step on one host core over the same scene."""
    n, x, y, m, p = c0_dam_break()
    params = vf.flip_params(*p)
    steps = 1000
    zeros = np.zeros_like(x)
    ms_by = {}
    for graph in (False, True):
        with vf.ParticleSimulation(n, n, len(x), tait=True, sticky=WALL_BATCH) as s:
            s.set_graph(graph)
            s.load(x, y, zeros, zeros, m, params)
            s.advance(20, 10)
            s.read("m")   # a blocking read: the device is idle
            t0 = time.perf_counter()
            s.advance(steps, 10)
            s.read("m")
            ms_by[graph] = 1e3 * (time.perf_counter() - t0)   # host clock: launches and the final read included
    ms = ms_by[False]
    cpu = None
    if not args.no_cpu and dist.rank == 0:
        sys.path.insert(0, str(ROOT / "tests"))
        from _oracle import Flip2State
        o = Flip2State(n, n, x, y, m)
        pw = np.array(params, np.float32)
        t0, done = time.perf_counter(), 0
        while time.perf_counter() - t0 < 2.0:
            if done % 10 == 0:
                o.sort()
            o.step(pw, (1, WALL_BATCH))
            done += 1
        el = time.perf_counter() - t0
        cpu = {"value": len(x) * done / el, "unit": "particle-steps/s", "cores": 1, "kind": "port",
               "sample": f"{done} steps of the same scene, oracle C port of FlipStep.step, 1 thread, {el:.1f} s"}
    return {"workload": "2D dam break 128^2 (config 0): 8192 particles, Tait k=50, sticky walls 3, dt 1e-4, sorted "
                        "every 10 steps; host-clock time of 1000 steps (launch-bound at this size)",
            "particles": len(x), "steps": steps, "ms_per_step": ms / steps,
            "particle_steps_per_s": len(x) * steps / (ms / 1e3),
            "graph": {"ms_per_step": ms_by[True] / steps, "particle_steps_per_s": len(x) * steps / (ms_by[True] / 1e3),
                      "how": "vf_mpm2_set_graph: a sort and the ten steps after it per graph launch"},
            "cpu_baseline": cpu}


def cpu_swe_rate(h, budget_s=10.0):
    """The oracle's shallow-water step (plain C, one thread) on the 4096^2 state: cell-updates/s."""
    sys.path.insert(0, str(ROOT / "tests"))
    from _oracle import OracleSweBackend, Stepper, swe_params
    n = N_SWE
    z = np.zeros_like(h)
    st = Stepper(OracleSweBackend(n, n, (0, 0, 0, 0)), n, n)
    st.set(h, z, z, swe_params(9.81, 0.45, 1.0, 1.0, 1e-6), 1e9)
    t0, done = time.perf_counter(), 0
    while done < 1 or time.perf_counter() - t0 < budget_s:
        st.step(1)
        done += 1
        if done >= 20:
            break
    el = time.perf_counter() - t0
    return {"value": n * n * done / el, "unit": "cell-updates/s", "cores": 1, "kind": "port",
            "sample": f"{done} steps of the same 4096^2 state, oracle C port of ShallowWater.kernel, 1 thread, "
                      f"{el:.1f} s"}


def run_literal(args, vf):
    """The 3D configuration's literal box, [0.05,0.65] in y: 12,734,496 particles, the same step, K device-timed steps."""
    x, y, z, m, params = dam3(BOX3_LITERAL)
    np3 = len(x)
    zeros = np.zeros(np3, np.float32)
    steps = min(args.steps, 50)
    with vf.ParticleSimulation3(N3, N3, N3, np3) as sim:
        sim.load([x, y, z], [zeros, zeros, zeros], m, vf.flip3_params(*params))
        sim.advance(3)
        sim.finish()
        e0, e1 = vf.Event(), vf.Event()
        e0.record(sim.stream())
        sim.advance(steps)
        e1.record(sim.stream())
        ms = e0.elapsed_ms(e1)
        sim.profile(True)
        sim.advance(steps)
        sim.finish()
        prof = sim.profile_read()
        sim.profile(False)
        touched = sim.touched_nodes()
    return {"workload": "3D dam break, the config's literal box [0.05,0.45]x[0.05,0.65]x[0.05,0.45] at 8 per cell",
            "particles": np3, "steps": steps, "ms_per_step": ms / steps,
            "particle_steps_per_s": np3 * steps / (ms / 1e3), "roofline": roofline3(prof, steps, np3, touched)}


def cpu_step_rate(x, y, z, m, params, budget_s=10.0, min_steps=10, max_steps=40, warmup=1):
    """The oracle's threaded 3D step on the host cores over the full workload: particle-steps/s over at least
    `min_steps` steps (more while the budget lasts), after `warmup` untimed steps."""
    sys.path.insert(0, str(ROOT / "tests"))
    from _oracle import Flip3State, OrPhysics, fp, lib as olib
    n = N3
    s = Flip3State(n, n, n, x, y, z, m)
    pw = np.ascontiguousarray(np.array(params, np.float32))
    threads = olib().or_baseline_threads()
    t0 = time.perf_counter()
    for _ in range(max(1, warmup)):   # warm-up (page faults)
        olib().or_flip3_step_omp(ctypes.byref(s.s), fp(pw), OrPhysics(0, 0), None)
    first = (time.perf_counter() - t0) / max(1, warmup)
    steps = max(min_steps, min(max_steps, int(budget_s / max(first, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(steps):
        olib().or_flip3_step_omp(ctypes.byref(s.s), fp(pw), OrPhysics(0, 0), None)
    el = time.perf_counter() - t0
    return len(x) * steps / el, threads, steps, el


# ---------------------------------------------------------------------------------------------- arms

METRIC = "MPM particle-steps/s"
DATA = "synthetic (seeded jittered dam break)"


def run_reference(args, dist: Dist):
    """The reference arm: the oracle's C restatement of Flip3Step (the reference's own CPU path cannot run here),
    OpenMP on all host threads, W untimed steps then K timed steps of the full workload, on rank 0 only."""
    if dist.rank != 0:
        return
    x, y, z, m, params = dam3()
    rate, threads, steps, el = cpu_step_rate(x, y, z, m, params, budget_s=0.0, min_steps=max(1, args.steps),
                                             max_steps=max(1, args.steps), warmup=max(1, args.warmup))
    sample = (f"{steps} full steps of the 8.16M-particle 256^3 workload after {max(1, args.warmup)} untimed ones "
              f"(oracle C port of Flip3Step, OpenMP, {threads} threads), {el:.1f} s")
    line = {"metric": METRIC, "value": rate, "unit": "particle-steps/s", "n_gpus": args.gpus,
            "steps": steps, "warmup": max(1, args.warmup), "ms_per_step": el / steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": DATA,
            "config": {"workload": WORKLOAD3, "particles": len(x), "grid": [N3] * 3},
            "impl": "reference",
            "cpu_baseline": {"value": rate, "unit": "particle-steps/s", "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": rate, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def emit(name, result, detail):
    """A sub-measurement: one JSON line on stdout (before the headline, which is always the last line), and the
    same object into the detail file when one is named."""
    if result is None:
        return
    print(json.dumps({"sub": name, **result}), flush=True)
    if detail is not None:
        detail[name] = result


def run_extras(args, vf, dist, sim=None):
    """The sub-measurements asked for with --only, each one JSON line on stdout."""
    detail = args.detail_store
    if "variants" in args.extras and sim is not None:
        emit("p2g_variants", run_variants(args, vf, sim), detail)
    peak, _ = measured_peaks()
    if "literal" in args.extras:
        emit("literal_box", run_literal(args, vf), detail)
    if "c0" in args.extras:
        emit("c0_2d", run_c0(args, vf, dist), detail)
    if "swe" in args.extras:
        emit("swe", run_swe(args, vf, dist, peak), detail)
    if "batch" in args.extras:
        emit("batch", run_batch(args, vf, dist, peak), detail)
    if "next" in args.extras:
        emit("next_rows", run_next_rows(args, vf, peak, cpu=not args.no_cpu and dist.rank == 0), detail)
    if "learned" in args.extras:
        emit("learned", run_learned(args, vf), detail)
    if "cnn" in args.extras:
        emit("cnn", run_cnn(args, vf), detail)
    if detail is not None and dist.rank == 0:
        pathlib.Path(args.detail).write_text(json.dumps(detail, indent=1))


def run_ours(args, dist: Dist):
    vf = package()
    vf.set_device(dist.local)
    if args.no_headline:
        run_extras(args, vf, dist)
        return
    x, y, z, m, params = dam3()
    np3 = len(x)
    zeros = np.zeros(np3, np.float32)
    sim = vf.ParticleSimulation3(N3, N3, N3, np3)
    sim.load([x, y, z], [zeros, zeros, zeros], m, vf.flip3_params(*params))
    stream = sim.stream()
    ev0, ev1 = vf.Event(), vf.Event()

    sim.advance(args.warmup)
    sim.finish()

    # timed region: K steps, device events on the handle's stream, barrier + sync on both sides
    dist.barrier()
    sim.finish()
    launches0 = sim.launches()
    with Clocks(dist.local) as clocks:
        ev0.record(stream)
        sim.advance(args.steps)
        ev1.record(stream)
        ms = ev0.elapsed_ms(ev1)
    sim.finish()
    launches = sim.launches() - launches0
    dist.barrier()
    ms_max = dist.max(ms)
    work = dist.sum(float(np3) * args.steps)
    value = work / (ms_max / 1e3)

    # per-kernel device times over a second, profiled run of K steps (events around every launch)
    sim.profile(True)
    sim.advance(args.steps)
    sim.finish()
    prof = sim.profile_read()
    sim.profile(False)
    touched = sim.touched_nodes()
    roof = roofline3(prof, args.steps, np3, touched)
    total_prof = sum(v[0] for v in prof.values())
    kernels = {k: round(v[0] / total_prof, 4) for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])[:4]}

    # end to end through the public API: pinned host arrays in (load), K steps, positions out (read)
    outs = [np.empty(np3, np.float32) for _ in range(3)]
    with vf.Pinned(*([x, y, z] + [zeros, m] + outs)):
        dist.barrier()
        sim.finish()
        ev0.record(stream)
        sim.load([x, y, z], [zeros, zeros, zeros], m, vf.flip3_params(*params))
        sim.advance(args.steps)
        for a, name in zip(outs, ("x", "y", "z")):
            vf.check(vf.lib().vf_mpm3_read(sim._h, vf.FIELDS3[name], vf._fp(a), np3))
        ev1.record(stream)
        e2e_ms = dist.max(ev0.elapsed_ms(ev1))
    e2e = {"value": dist.sum(float(np3) * args.steps) / (e2e_ms / 1e3), "unit": "particle-steps/s",
           "h2d_bytes_per_step": 7 * np3 * 4 / args.steps, "d2h_bytes_per_step": 3 * np3 * 4 / args.steps,
           "job": f"load 7 fields + {args.steps} steps + read x,y,z"}
    if "variants" in args.extras:
        run_extras(args, vf, dist, sim)
        args.extras = args.extras - {"variants"}
    sim.close()
    run_extras(args, vf, dist)

    if dist.rank != 0:
        return
    cpu = None
    if not args.no_cpu:
        rate, threads, cpu_steps, cpu_el = cpu_step_rate(x, y, z, m, params)
        cpu = {"value": rate, "unit": "particle-steps/s", "cores": threads, "kind": "port",
               "sample": f"{cpu_steps} full steps of this workload, oracle C port of Flip3Step, OpenMP, {cpu_el:.1f} s"}
    line = {
        "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": DATA,
        "config": {"workload": WORKLOAD3, "particles": np3, "grid": [N3] * 3, "parallelism": f"replicas x{dist.world}",
                   "l2": "inputs larger than L2 (particles 555 MB a set)"},
        "roofline": roof,
        "kernels_share": kernels,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clocks.summary(),
    }
    text = json.dumps(line)
    assert len(text) < 2048, f"the headline line grew to {len(text)} bytes"
    print(text, flush=True)


def roofline3(prof, steps, np3, touched):
    """The roofline of the step's dominant kernel from a profiled run (CUDA events around every launch).

    Separate passes (the default): k_p2g3_tile + k_g2p3_tile at 152 Np + 28 N_t.
    Fused step (opt-in): k_g2p2g3 gathers each particle from grid k and scatters it into grid k+1, so the P2G+G2P
    pair is one kernel. Its algorithmic bytes a launch: read x, y, z, m, j (20 B) and write the 16 advected fields
    (64 B) a particle, read grid k's four floats and write grid k+1's four floats a touched node (32 B): 84 Np + 32 N_t.
    `pair_target_ms` is the time the separate passes' bytes (152 Np + 28 N_t) take at 70% of the peak: the P2G+G2P
    target at 8M particles, which either form's time is compared with."""
    peak, peak_kind = measured_peaks()
    sep_bytes = 152.0 * np3 + 28.0 * touched
    if "k_g2p2g3" in prof:
        t, n = prof["k_g2p2g3"]
        per_ms = t / n
        alg = 84.0 * np3 + 32.0 * touched
        kernel, tr = "k_g2p2g3 (fused G2P of step k + P2G of step k+1)", profiled_traffic("k_g2p2g3")
    else:
        t_p2g = prof.get("k_p2g3_tile", (0.0, 1))
        t_g2p = prof.get("k_g2p3_tile", (0.0, 1))
        per_ms = (t_p2g[0] + t_g2p[0]) / steps
        alg = sep_bytes
        tr_p2g, tr_g2p = profiled_traffic("k_p2g3_tile"), profiled_traffic("k_g2p3_tile")
        tr = (tr_p2g + tr_g2p) if (tr_p2g is not None and tr_g2p is not None) else None
        kernel = "k_p2g3_tile + k_g2p3_tile"
    achieved = alg / (per_ms / 1e3) / 1e9
    return {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": tr, "kernel": kernel, "peak_kind": peak_kind,
            "algorithmic_bytes": alg, "touched_nodes": touched, "pair_ms": round(per_ms, 4),
            "pair_target_ms": round(sep_bytes / (0.7 * peak * 1e9) * 1e3, 4)}


def run_variants(args, vf, sim):
    """The P2G schedules the 3D configuration compares, each for K profiled steps from the same state."""
    ev0, ev1 = vf.Event(), vf.Event()
    stream = sim.stream()
    variants = {}
    names = {vf.VF_P2G_ATOMIC: "global_atomic", vf.VF_P2G_WARP: "warp_aggregated", vf.VF_P2G_TILE: "sorted_smem_tile",
             vf.VF_P2G_FIXED: "exact_fixed_point", -1: "sorted_smem_tile_fused"}
    for sched in (vf.VF_P2G_ATOMIC, vf.VF_P2G_WARP, vf.VF_P2G_FIXED, vf.VF_P2G_TILE, -1):
        sim.set_schedule(vf.VF_P2G_TILE if sched < 0 else sched)
        sim.set_fused(sched < 0)
        sim.advance(2)
        sim.finish()
        sim.profile(True)
        ev0.record(stream)
        sim.advance(args.variant_steps)
        ev1.record(stream)
        v_ms = ev0.elapsed_ms(ev1)
        vp = sim.profile_read()
        sim.profile(False)
        p2g = [k for k in vp if k.startswith("k_p2g3") or k == "k_fixed_to_grid3"]
        variants[names[sched]] = {
            "ms_per_step": v_ms / args.variant_steps,
            "p2g_ms_per_step": sum(vp[k][0] for k in p2g) / args.variant_steps,
            "kernels_ms_per_step": {k: v[0] / args.variant_steps for k, v in vp.items()}}
    sim.set_schedule(vf.VF_P2G_TILE)
    sim.set_fused(True)
    return {"workload": WORKLOAD3, "steps": args.variant_steps, "schedules": variants}


def run_swe(args, vf, dist, peak):
    """Shallow water, 4096^2 HLL: cell-updates/s and the tile kernel's roofline at 24 B a cell, in the exact
    arithmetic (bit for bit the reference's) and in the fast mode; the oracle on one core as the CPU baseline."""
    h = swe_bumps(args.swe_n)
    zero2 = np.zeros_like(h)
    ev0, ev1 = vf.Event(), vf.Event()
    n = args.swe_n
    cells = n * n
    out = {"workload": f"HLL shallow water {n}^2, dx=1, 16 seeded bumps, walls, C=0.45 (config 2 at 4096^2)"}
    for exact in (True, False):
        with vf.PatchSimulation(n, n) as p:
            p.set_exact(exact)
            p.load(h, zero2, zero2, vf.swe_params(9.81, 0.45, 1.0, 1.0, 1e-6))
            p.write_budget(0, 2 ** 31 - 1)
            p.dispatch(3)
            p.read_budget(0)
            k_swe = max(10, args.steps)
            s_stream = p.stream()
            ev0.record(s_stream)
            p.dispatch(k_swe)
            ev1.record(s_stream)
            swe_ms = ev0.elapsed_ms(ev1)
            p.profile(True)
            p.dispatch(k_swe)
            p.read_budget(0)
            sp = p.profile_read()
            p.profile(False)
        name = "k_swe_tile" if exact else "k_swe_strip_fast"
        k_ms = sp[name][0] / sp[name][1]
        achieved = 24.0 * cells / (k_ms / 1e3) / 1e9
        out["exact" if exact else "fast"] = {
            "steps": k_swe, "cell_updates_per_s": cells * k_swe / (swe_ms / 1e3), "ms_per_step": swe_ms / k_swe,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "kernel": name, "bytes_per_cell": 24}}
    out["cpu_baseline"] = None if (args.no_cpu or dist.rank != 0 or n != N_SWE) else cpu_swe_rate(h)
    return out


CNN_FLOPS_PER_CELL = 2 * 25 * (3 * 32 + 32 * 32 + 32 * 6)   # 65.6 kFLOP: the three convolutions, algorithmic


def timed_steps(vf, sim, steps):
    """ms per step of `steps` steps on the handle's stream, then the same steps profiled per kernel."""
    ev0, ev1 = vf.Event(), vf.Event()
    sim.advance(3)
    sim.finish()
    ev0.record(sim.stream())
    sim.advance(steps)
    ev1.record(sim.stream())
    ms = ev0.elapsed_ms(ev1) / steps
    sim.profile(True)
    sim.advance(steps)
    sim.finish()
    prof = {k: v[0] / steps for k, v in sim.profile_read().items()}
    sim.profile(False)
    return ms, prof


def plain_ms(vf, sim, steps):
    """ms per step of `steps` steps on the handle's stream, after ten untimed ones (a replayed run captures its
    graph within them)."""
    ev0, ev1 = vf.Event(), vf.Event()
    sim.advance(10)
    sim.finish()
    ev0.record(sim.stream())
    sim.advance(steps)
    ev1.record(sim.stream())
    ms = ev0.elapsed_ms(ev1) / steps
    sim.finish()
    return ms


TENSION_KERNELS = {"k_tension3_colour": 8.0, "k_tension3_blur": 8.0 * 5, "k_tension3_stress": 28.0,
                   "k_grid3_tension": 60.0}   # algorithmic bytes per node per step (5 blur launches)


def cpu_tension_rate(n, x, y, z, m, params, tension, budget_s, max_steps):
    """The oracle's threaded 3D step (with tension's passes if asked) on the host cores: particle-steps/s."""
    sys.path.insert(0, str(ROOT / "tests"))
    from _oracle import Flip3State, OrPhysics, fp, lib as olib
    s = Flip3State(n, n, n, x, y, z, m)
    pw = np.ascontiguousarray(np.array(params, np.float32))
    scratch = np.zeros(8 * n ** 3, np.float32) if tension else None

    def step():
        if tension:
            olib().or_flip3_step_tension_omp(ctypes.byref(s.s), fp(pw), OrPhysics(0, 0), None, fp(scratch))
        else:
            olib().or_flip3_step_omp(ctypes.byref(s.s), fp(pw), OrPhysics(0, 0), None)

    t0 = time.perf_counter()
    step()   # warm-up (page faults)
    first = time.perf_counter() - t0
    steps = max(1, min(max_steps, int(budget_s / max(first, 1e-4))))
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    el = time.perf_counter() - t0
    return {"value": len(x) * steps / el, "unit": "particle-steps/s", "cores": olib().or_baseline_threads(),
            "kind": "port", "sample": f"{steps} steps of the same workload, oracle C port of Flip3Step"
                                      f"{' with tension' if tension else ''}, OpenMP, {el:.1f} s"}


def run_next_rows(args, vf, peak, cpu=False):
    """Surface tension on the 3D configuration, and sparse storage on it and on a blob in a wide domain."""
    x, y, z, m, params = dam3()
    np3 = len(x)
    zeros = np.zeros(np3, np.float32)
    nodes = N3 ** 3
    steps = args.variant_steps
    out = {}
    sigma = 0.01 * params[4]
    with vf.ParticleSimulation3(N3, N3, N3, np3, tension=True) as sim:
        sim.load([x, y, z], [zeros, zeros, zeros], m, vf.flip3_params(*params, sigma))
        ms, prof = timed_steps(vf, sim, steps)
    t_ms = sum(prof.get(k, 0.0) for k in TENSION_KERNELS)
    t_bytes = sum(TENSION_KERNELS.values()) * nodes
    out["tension"] = {
        "workload": f"{WORKLOAD3}, with Tension3's passes (sigma {sigma:.4g})", "steps": steps,
        "ms_per_step": ms, "particle_steps_per_s": np3 / (ms / 1e3), "tension_ms_per_step": t_ms,
        "roofline": {"bound": "hbm", "kernels": sorted(TENSION_KERNELS), "bytes_per_node": sum(TENSION_KERNELS.values()),
                     "achieved": t_bytes / (t_ms / 1e3) / 1e9, "peak": peak,
                     "frac": t_bytes / (t_ms / 1e3) / 1e9 / peak, "unit": "GB/s"},
        "kernels_ms_per_step": prof,
        "cpu_baseline": cpu_tension_rate(N3, x, y, z, m, (*params, sigma), True, 10.0, 8) if cpu else None}

    # the same configuration with advance() replayed from a captured two-step graph
    with vf.ParticleSimulation3(N3, N3, N3, np3) as sim:
        sim.set_graph(True)
        sim.load([x, y, z], [zeros, zeros, zeros], m, vf.flip3_params(*params))
        ms = plain_ms(vf, sim, steps)
    out["graph_config"] = {"workload": WORKLOAD3, "steps": steps, "ms_per_step": ms,
                           "particle_steps_per_s": np3 / (ms / 1e3)}
    # the reference's scale: Tension3Test's drop (radius 8 in a 40^3 box), launched kernel by kernel and replayed
    rng = np.random.default_rng(7)
    c = np.argwhere(np.ones((16, 16, 16), bool)).astype(np.float32) + np.float32(12)
    c = c[((c + 0.5 - 20.0) ** 2).sum(1) <= 64.0]
    pos = np.repeat(c, PPC3, axis=0) + rng.random((len(c) * PPC3, 3), dtype=np.float32) * np.float32(0.999)
    sx, sy, sz = (np.ascontiguousarray(pos[:, a], np.float32) for a in range(3))
    sm = np.full(len(sx), np.float32(1.0 / PPC3), np.float32)
    s0 = np.zeros_like(sx)
    bulk_s = 200.0 ** 2
    small = {"workload": f"a drop of radius 8 ({len(sx)} particles) at rest in a 40^3 box, no gravity (Tension3Test)",
             "steps": 400}
    for tension in (False, True):
        for graph in (False, True):
            with vf.ParticleSimulation3(40, 40, 40, len(sx), tension=tension) as sim:
                sim.set_graph(graph)
                sim.load([sx, sy, sz], [s0, s0, s0], sm,
                         vf.flip3_params(0.3 / 220.0, 0.0, 0.0, 0.0, bulk_s, 1.0, 0.08 * bulk_s if tension else 0.0))
                ms = plain_ms(vf, sim, 400)
            small[f"{'tension' if tension else 'plain'}_{'graph' if graph else 'launched'}_ms_per_step"] = ms
        if cpu:
            small[f"{'tension' if tension else 'plain'}_cpu_baseline"] = cpu_tension_rate(
                40, sx, sy, sz, sm, (0.3 / 220.0, 0.0, 0.0, 0.0, bulk_s, 1.0, 0.08 * bulk_s if tension else 0.0),
                tension, 3.0, 400)
    names = {vf.VF_P2G_TILE: "tile", vf.VF_P2G_ATOMIC: "atomic", vf.VF_P2G_WARP: "warp", vf.VF_P2G_AUTO: "auto"}
    for sched in names:
        with vf.ParticleSimulation3(40, 40, 40, len(sx), schedule=sched) as sim:
            sim.set_graph(True)
            sim.load([sx, sy, sz], [s0, s0, s0], sm, vf.flip3_params(0.3 / 220.0, 0.0, 0.0, 0.0, bulk_s, 1.0))
            small[f"plain_graph_{names[sched]}_ms_per_step"] = plain_ms(vf, sim, 400)
            _, prof = timed_steps(vf, sim, 100)
            small[f"plain_{names[sched]}_kernels_ms_per_step"] = {k: round(v, 5) for k, v in prof.items()}
    out["small_scene"] = small

    sparse = {}
    pages = (N3 // 8) ** 3
    with vf.ParticleSimulation3(N3, N3, N3, np3, pool_bricks=pages) as sim:
        sim.load([x, y, z], [zeros, zeros, zeros], m, vf.flip3_params(*params))
        ms, prof = timed_steps(vf, sim, steps)
        used = sim.pool_used()
    sparse["config"] = {"workload": WORKLOAD3, "steps": steps, "ms_per_step": ms,
                        "particle_steps_per_s": np3 / (ms / 1e3), "pool_bricks": pages, "bricks_used": used,
                        "p2g_g2p_ms_per_step": prof.get("k_p2g3_tile", 0.0) + prof.get("k_g2p3_tile", 0.0)}
    # a ball of water (radius 24 nodes) falling in the middle of the same 256^3 domain
    rng = np.random.default_rng(5)
    c = np.argwhere(np.ones((48, 48, 48), bool)).astype(np.float32) + np.float32(104)
    c = c[((c + 0.5 - 128.0) ** 2).sum(1) <= 24.0 ** 2]
    pos = (np.repeat(c, PPC3, axis=0) + rng.random((len(c) * PPC3, 3), dtype=np.float32) * np.float32(0.999))
    bx, by, bz = (np.ascontiguousarray(pos[:, a], np.float32) for a in range(3))
    bm = np.full(len(bx), np.float32(1.0 / PPC3), np.float32)
    bz0 = np.zeros_like(bx)
    blob = {"workload": f"a ball of radius 24 nodes ({len(bx)} particles, 8 per cell) falling in a {N3}^3 domain",
            "steps": steps}
    for name, kw in (("dense", {}), ("sparse", {"pool_bricks": 512})):
        with vf.ParticleSimulation3(N3, N3, N3, len(bx), **kw) as sim:
            sim.load([bx, by, bz], [bz0, bz0, bz0], bm, vf.flip3_params(*params))
            ms, _ = timed_steps(vf, sim, steps)
            blob[name] = {"ms_per_step": ms, "particle_steps_per_s": len(bx) / (ms / 1e3),
                          "grid_bytes": 2 * (512 * 512 * 16 if kw else nodes * 16)}
            if kw:
                blob[name]["bricks_used"] = sim.pool_used()
    sparse["blob"] = blob
    # many blobs in one pool (the reference's planned experiment): n balls of radius 8 spread through a 256^3 domain
    # and stepped together, against the same balls as n separate 40^3 boxes stepped one after another
    drop = np.argwhere(np.ones((16, 16, 16), bool)).astype(np.float32)
    drop = drop[((drop + 0.5 - 8.0) ** 2).sum(1) <= 64.0]
    many = {"workload": "n balls of radius 8 (1,704 cells, 8 particles each) in one 256^3 domain with sparse storage, "
                        "against n separate 40^3 boxes (VF_P2G_AUTO, graph replay)", "steps": 100}
    for nb in (1, 4, 16):
        sites = [(48 + 48 * (k % 4), 48 + 48 * ((k // 4) % 4), 128) for k in range(nb)]
        cells = np.concatenate([drop + np.array(c, np.float32) - 8.0 for c in sites])
        pos = np.repeat(cells, PPC3, axis=0) + rng.random((len(cells) * PPC3, 3), dtype=np.float32) * np.float32(0.999)
        mx, my, mz = (np.ascontiguousarray(pos[:, a], np.float32) for a in range(3))
        mm = np.full(len(mx), np.float32(1.0 / PPC3), np.float32)
        m0 = np.zeros_like(mx)
        with vf.ParticleSimulation3(N3, N3, N3, len(mx), pool_bricks=64 * nb) as sim:
            sim.set_graph(True)
            sim.load([mx, my, mz], [m0, m0, m0], mm, vf.flip3_params(*params))
            pooled = plain_ms(vf, sim, 100)
            used = sim.pool_used()
        one = len(drop) * PPC3
        boxes = []
        for k in range(nb):
            sl = slice(k * one, (k + 1) * one)
            b = vf.ParticleSimulation3(40, 40, 40, one, schedule=vf.VF_P2G_AUTO)
            b.set_graph(True)
            off = np.array(sites[k], np.float32) - 20.0
            b.load([mx[sl] - off[0], my[sl] - off[1], mz[sl] - off[2]], [m0[sl]] * 3, mm[sl], vf.flip3_params(*params))
            b.advance(10)   # the graph is captured here, not in the timed steps
            b.finish()
            boxes.append(b)
        t0 = time.perf_counter()
        for b in boxes:   # each box on its own stream, so their steps may overlap on the device
            b.advance(100)
        for b in boxes:
            b.finish()
        separate = 1e3 * (time.perf_counter() - t0) / 100   # host clock over all boxes' streams
        for b in boxes:
            b.close()
        many[str(nb)] = {"pool_ms_per_step": pooled, "bricks_used": used, "separate_boxes_ms_per_step": separate}
    sparse["many_blobs"] = many
    out["sparse"] = sparse
    return out


def run_learned(args, vf):
    """The learned coarse shallow-water configuration: the committed network (trained at 2048^2 on held-in seeds)
    against the plain fine solver and the plain coarse solver on held-out seeds, 2000 fine steps each."""
    from vexfluid import learned as L
    net, report = L.trained()
    seeds = list(range(1, 1 + args.learned_seeds))
    rows = []
    try:
        for seed in seeds:
            rows.append(L.evaluate_pair(net, report["fine"], seed, 2000, report["interval_ticks"]))
        # the network's kernels, timed alone over a few corrections of the coarse grid
        with vf.PatchSimulation(report["coarse"], report["coarse"]) as c:
            h0 = L.restrict(L.bumps(3, report["fine"]))
            z = np.zeros_like(h0)
            c.load(h0.ravel(), z.ravel(), z.ravel(), L.coarse_params())
            net.correct(c)
            net.profile(True)
            for _ in range(10):
                net.correct(c)
            prof = net.profile_read()
            net.profile(False)
    finally:
        net.close()
    conv_ms = sum(prof[k][0] / prof[k][1] for k in ("k_conv1", "k_conv2", "k_conv3"))
    cells = report["coarse"] ** 2
    tflops = CNN_FLOPS_PER_CELL * cells / (conv_ms / 1e3) / 1e12
    tpeak, tkind = measured_tensor_peak()
    mean = lambda key, k: float(np.mean([r[k][key] for r in rows]))
    return {
        "workload": (f"learned coarse shallow water: fine {report['fine']}^2 HLL (16 bumps, the 4096^2 distribution "
                     f"halved in sigma and centres), coarse {report['coarse']}^2, correction every "
                     f"{report['interval_coarse_steps']} coarse steps ({report['interval_ticks']} ticks), "
                     f"held-out seeds {seeds[0]}..{seeds[-1]}, 2000 fine steps each"),
        "fine_cell_updates_per_s": mean("fine_cell_updates_per_s", 1),
        "learned_equivalent_cell_updates_per_s": mean("equivalent_fine_cell_updates_per_s", 1),
        "speedup_vs_fine": mean("speedup", 1),
        "speedup_min_max": [float(min(r[1]["speedup"] for r in rows)), float(max(r[1]["speedup"] for r in rows))],
        "plain_coarse_speedup_vs_fine": mean("speedup", 0),
        "h_rms_error": {"learned": mean("h_rms_error", 1), "plain_coarse": mean("h_rms_error", 0),
                        "learned_max": float(max(r[1]["h_rms_error"] for r in rows))},
        "per_seed": [{"seed": r[0]["seed"], "plain_err": r[0]["h_rms_error"], "learned_err": r[1]["h_rms_error"],
                      "speedup": r[1]["speedup"]} for r in rows],
        "network_kernels_us": {k: 1e3 * v[0] / v[1] for k, v in prof.items()},
        "roofline": {"bound": "tensor", "achieved": tflops, "peak": tpeak, "unit": "TFLOP/s", "frac": tflops / tpeak,
                     "peak_kind": tkind, "traffic": None, "kernel": "k_conv1 + k_conv2 + k_conv3 (tcgen05), bf16",
                     "flops_per_cell": CNN_FLOPS_PER_CELL},
        "training": {"seeds": report["train_seeds"], "pairs_per_seed": report["pairs_per_seed"],
                     "adam_steps": report["adam_steps"], "train_seconds": report["train_seconds"]},
    }


def run_cnn(args, vf):
    """The flux network alone: the committed network corrects a 1024^2 coarse patch (a restricted bump state)
    three times; the per-kernel device times of the corrections and the convolutions' tensor roofline."""
    from vexfluid import learned as L
    net, report = L.trained()
    try:
        with vf.PatchSimulation(report["coarse"], report["coarse"]) as c:
            h0 = L.restrict(L.bumps(3, report["fine"]))
            z = np.zeros_like(h0)
            c.load(h0.ravel(), z.ravel(), z.ravel(), L.coarse_params())
            net.correct(c)
            net.profile(True)
            for _ in range(3):
                net.correct(c)
            prof = net.profile_read()
            net.profile(False)
    finally:
        net.close()
    conv_ms = sum(prof[k][0] / prof[k][1] for k in ("k_conv1", "k_conv2", "k_conv3"))
    cells = report["coarse"] ** 2
    tflops = CNN_FLOPS_PER_CELL * cells / (conv_ms / 1e3) / 1e12
    tpeak, tkind = measured_tensor_peak()
    return {"workload": f"flux network corrections of a {report['coarse']}^2 coarse patch",
            "network_kernels_us": {k: 1e3 * v[0] / v[1] for k, v in prof.items()},
            "roofline": {"bound": "tensor", "achieved": tflops, "peak": tpeak, "unit": "TFLOP/s",
                         "frac": tflops / tpeak, "peak_kind": tkind, "flops_per_cell": CNN_FLOPS_PER_CELL}}


def cpu_batch_rate(scenes, x, y, m, budget_s=10.0):
    """The oracle's 2D step, one scene after another on one host core, over the first scenes of the batch
    until the budget is spent: particle-steps/s."""
    sys.path.insert(0, str(ROOT / "tests"))
    from _oracle import Flip2State
    done, spent, at, used = 0, 0.0, 0, 0
    for n, count, params in scenes:
        s = Flip2State(n, n, x[at:at + count], y[at:at + count], m[at:at + count])
        pw = np.array(params, np.float32)
        t0 = time.perf_counter()
        s.step(pw, (1, WALL_BATCH))
        s.step(pw, (1, WALL_BATCH))
        spent += time.perf_counter() - t0
        done += 2 * count
        at += count
        used += 1
        if spent > budget_s:
            break
    return done / spent, used, spent


def run_batch(args, vf, dist: Dist, peak):
    """The batched 2D config: 256 dam-break scenes in one cooperative launch per step, replayed from CUDA graphs,
    tiles and block size from the autotuner (its JSON cache). Scenes are dealt round-robin to the ranks."""
    scenes, x, y, m = batch_scenes()
    first = np.concatenate([[0], np.cumsum([c for _, c, _ in scenes])])
    mine = list(range(dist.rank, len(scenes), dist.world))
    table = [vf.Scene(n, n, c, vf.flip_params(*p)) for n, c, p in (scenes[k] for k in mine)]
    pick = lambda a: [a[first[k]:first[k + 1]] for k in mine]
    xs, ys, ms = pick(x), pick(y), pick(m)
    zs = [np.zeros_like(a) for a in xs]
    nparts = sum(len(a) for a in xs)
    t0 = time.perf_counter()
    table, block, trials = vf.autotune(table, xs, ys, zs, zs, ms, tait=True, sticky=WALL_BATCH,
                                       cache=args.tune_cache)
    tune_s = time.perf_counter() - t0
    b = vf.BatchSimulation(table, tait=True, sticky=WALL_BATCH, block=block)
    b.load(xs, ys, zs, zs, ms)
    b.advance(max(3, args.warmup))
    b.finish()
    b.phases()
    k = max(32, args.steps)
    ev0, ev1 = vf.Event(), vf.Event()
    stream = b.stream()
    dist.barrier()
    launches0 = b.launches()
    ev0.record(stream)
    b.advance(k)
    ev1.record(stream)
    ms = ev0.elapsed_ms(ev1)
    b.finish()
    launches = b.launches() - launches0
    ms_max = dist.max(ms)
    total = dist.sum(float(nparts))
    ph = b.phases()   # the kernel's own per-phase clock over the timed steps
    nl = max(1, ph.pop("launches"))
    phases = {k: v / nl for k, v in ph.items()}
    touched = 0
    for s in range(len(table)):
        touched += int(np.count_nonzero(b.read(s, "gm")))
    touched = dist.sum(float(touched))
    cfg = b.config(0)
    tiles = {}
    for s in table:
        tiles[f"{s.tile[0]}x{s.tile[1]}"] = tiles.get(f"{s.tile[0]}x{s.tile[1]}", 0) + 1
    b.close()
    # P2G reads 10 f32 per particle and writes m, mu, mv per touched node; G2P reads x, y, m, j and writes 10
    # f32 per particle and reads m, mu, mv per touched node: 96 Np + 24 N_t, over the whole step's time
    alg = 96.0 * total + 24.0 * touched
    achieved = alg / (ms_max / k / 1e3) / 1e9
    out = {"workload": (f"{N_BATCH} 2D dam-break scenes (seed {SEED_BATCH}), grids uniform over {BATCH_GRIDS}^2, "
                        f"particles log-uniform in [{BATCH_NP[0]}, {BATCH_NP[1]}], 4 per cell where the box fits, "
                        f"Tait k=50 m^2/s^2, rho0=1, sticky walls {WALL_BATCH}, dt 1e-4 (Courant-capped on 512^2)"),
           "scenes": len(scenes), "particles": int(total), "steps": k, "ms_per_step": ms_max / k,
           "particle_steps_per_s": total * k / (ms_max / 1e3), "launches_per_step": launches / k,
           "block": cfg["block"], "ctas": cfg["ctas"], "tiles": tiles, "tuner_trials": trials,
           "phases_ms_per_step": phases,
           "tuner_s": tune_s,
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                        "frac": achieved / peak, "traffic": None, "kernel": "k_batch2_step (whole step)",
                        "algorithmic_bytes_per_step": alg, "touched_nodes": touched}}
    if dist.rank == 0 and not args.no_cpu:
        rate, used, spent = cpu_batch_rate(scenes, x, y, m)
        out["cpu_baseline"] = {"value": rate, "unit": "particle-steps/s", "cores": 1, "kind": "port",
                               "sample": f"2 steps of each of the first {used} scenes, one after another, "
                                         f"oracle C port of FlipStep.step, 1 thread, {spent:.1f} s"}
    return out


EXTRAS = ("swe", "c0", "literal", "batch", "learned", "cnn", "variants", "next")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline legs")
    ap.add_argument("--only", default="",
                    help="comma-separated sub-measurements to run before the headline: " + ",".join(EXTRAS) +
                         " (or 'all'); each prints one JSON line, the headline stays the last line")
    ap.add_argument("--detail", default=None, help="also write the sub-measurements to this JSON file")
    ap.add_argument("--no-headline", action="store_true",
                    help="run only the --only sub-measurements (for profiling one of them), no headline line")
    ap.add_argument("--variant-steps", type=int, default=20)
    ap.add_argument("--swe-n", type=int, default=N_SWE, help="the shallow-water sub-measurement's grid side")
    ap.add_argument("--learned-seeds", type=int, default=64, help="held-out seeds of the learned evaluation")
    ap.add_argument("--tune-cache", default=str(PKG / "batch2_tune.json"),
                    help="the batched step's autotune cache (JSON)")
    args = ap.parse_args()
    wanted = {w.strip() for w in args.only.split(",") if w.strip()}
    if "all" in wanted:
        wanted = set(EXTRAS)
    unknown = wanted - set(EXTRAS)
    if unknown:
        ap.error(f"unknown sub-measurements: {sorted(unknown)}")
    args.extras = wanted
    args.detail_store = {} if args.detail else None
    dist = Dist()
    try:
        if args.impl == "reference":
            run_reference(args, dist)
        else:
            run_ours(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
