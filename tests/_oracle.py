"""ctypes bindings to the oracle (oracle/liboracle.so) and the reference tests' input generators.

Test infrastructure: the oracle is the CPU restatement of the reference step, and the
tests only ever check results against it. The generators regenerate the reference tests' seeded
inputs through a java.util.Random restatement:

* ``JavaRandom``          -- java.util.Random (Java SE API specification), pure Python.
* ``flip_column``         -- FlipTest.column (FlipTest.java:134-150).
* ``slab3``               -- Flip3Test's dam-break slab (Flip3Test.java:143-166).
* ``Particles.jittered``  -- ScatterTest.Particles.jittered/shuffled/sortedByCell
                             (ScatterTest.java:460-518).
"""
from __future__ import annotations

import ctypes
import math
import os
import pathlib
import subprocess
from dataclasses import dataclass

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[1]
ORACLE_DIR = ROOT / "oracle"
_LIB = None

f32p = ctypes.POINTER(ctypes.c_float)
f64p = ctypes.POINTER(ctypes.c_double)
i32p = ctypes.POINTER(ctypes.c_int32)
i64p = ctypes.POINTER(ctypes.c_int64)


class OrPhysics(ctypes.Structure):
    _fields_ = [("eos", ctypes.c_int), ("sticky", ctypes.c_int)]


class OrFlip2(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("np", ctypes.c_int)] + [
        (n, f32p) for n in ("x", "y", "u", "v", "m", "j", "c00", "c01", "c10", "c11", "gm", "gmu", "gmv", "gu", "gv")
    ]


class OrFlip3(ctypes.Structure):
    _fields_ = (
        [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("np", ctypes.c_int)]
        + [(n, f32p) for n in ("x", "y", "z", "u", "v", "w", "m", "j")]
        + [("c", f32p * 9)]
        + [(n, f32p) for n in ("gm", "gmu", "gmv", "gmw", "gu", "gv", "gw")]
    )


class OrSweDiag(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("volume", "min_depth", "max_depth", "max_speed", "max_froude",
                                              "max_courant")] + [(n, ctypes.c_int32) for n in
                                                                 ("non_finite", "negative", "wet")]


class OrParticleDiag(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("min_density", "max_density", "low_density", "high_density",
                                              "mach", "courant")] + [("non_finite", ctypes.c_int32)]


def lib():
    """The oracle library, built on first use if it is missing."""
    global _LIB
    if _LIB is None:
        so = ORACLE_DIR / "liboracle.so"
        if not so.exists():
            subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)
        L = ctypes.CDLL(str(so))
        L.or_flip2_step.argtypes = [ctypes.POINTER(OrFlip2), f32p, OrPhysics]
        L.or_flip2_step_relaxing.argtypes = [ctypes.POINTER(OrFlip2), f32p, OrPhysics]
        for n in ("or_flip2_scatter", "or_flip2_grid"):
            getattr(L, n).argtypes = [ctypes.POINTER(OrFlip2), f32p, OrPhysics]
        L.or_flip2_clear.argtypes = [ctypes.POINTER(OrFlip2)]
        L.or_flip2_advect.argtypes = [ctypes.POINTER(OrFlip2), f32p]
        L.or_flip2_sort.argtypes = [ctypes.POINTER(OrFlip2), i32p, i32p, f32p]
        L.or_cell2.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_int]
        L.or_cell2.restype = ctypes.c_int32
        L.or_sort2_keys.argtypes = [f32p, f32p, ctypes.c_int64, ctypes.c_int, ctypes.c_int, i32p]
        L.or_counting_sort.argtypes = [i32p, ctypes.c_int64, ctypes.c_int64, i32p, i32p]
        L.or_scatter2_bilinear.argtypes = [ctypes.c_int, ctypes.c_int] + [f32p] * 5 + [ctypes.c_int64] + [f32p] * 3
        L.or_scatter2_bilinear_f64.argtypes = [ctypes.c_int, ctypes.c_int] + [f32p] * 5 + [ctypes.c_int64] + [f64p] * 3
        L.or_cell_starts2.argtypes = [f32p, f32p, ctypes.c_int64, ctypes.c_int, ctypes.c_int, i32p, i64p]
        L.or_cell_starts2.restype = ctypes.c_int32
        L.or_fixed_scatter2.argtypes = [ctypes.c_int, ctypes.c_int] + [f32p] * 5 + [ctypes.c_int64, ctypes.c_int,
                                                                                  ctypes.c_int] + [i32p] * 3
        for n in ("or_flip3_step", "or_flip3_scatter", "or_flip3_grid"):
            getattr(L, n).argtypes = [ctypes.POINTER(OrFlip3), f32p, OrPhysics]
        L.or_fixed_scatter3.argtypes = [ctypes.POINTER(OrFlip3), f32p, OrPhysics, i64p]
        L.or_tension3_blur.argtypes = [ctypes.c_int] * 3 + [f32p, f32p, f32p, ctypes.c_int]
        L.or_tension3_colour.argtypes = [ctypes.c_int] * 3 + [f32p] * 4
        L.or_tension3_colour.restype = f32p
        L.or_tension3_stress.argtypes = [ctypes.c_int] * 3 + [f32p, f32p]
        L.or_flip3_grid_tension.argtypes = [ctypes.POINTER(OrFlip3), f32p, OrPhysics, f32p, f32p]
        L.or_flip3_step_tension.argtypes = [ctypes.POINTER(OrFlip3), f32p, OrPhysics, f32p]
        L.or_flip3_clear.argtypes = [ctypes.POINTER(OrFlip3)]
        L.or_flip3_advect.argtypes = [ctypes.POINTER(OrFlip3), f32p]
        L.or_flip3_sort.argtypes = [ctypes.POINTER(OrFlip3), i32p, i32p, i32p, f32p]
        L.or_flip3_step_omp.argtypes = [ctypes.POINTER(OrFlip3), f32p, OrPhysics, f32p]
        L.or_flip3_step_tension_omp.argtypes = [ctypes.POINTER(OrFlip3), f32p, OrPhysics, f32p, f32p]
        L.or_baseline_threads.restype = ctypes.c_int
        L.or_key3.argtypes = [ctypes.c_float] * 3 + [ctypes.c_int] * 3
        L.or_key3.restype = ctypes.c_int32
        L.or_key3_count.argtypes = [ctypes.c_int] * 3
        L.or_key3_count.restype = ctypes.c_int64
        swe = [ctypes.c_int, ctypes.c_int, i32p, f32p] + [f32p] * 6 + [i32p] * 6
        L.or_swe_dispatch.argtypes = swe
        L.or_swe_dispatch_omp.argtypes = swe
        L.or_swe_fastest_wave.argtypes = [f32p, f32p, f32p, ctypes.c_int64, ctypes.c_double, ctypes.c_double]
        L.or_swe_fastest_wave.restype = ctypes.c_int32
        L.or_swe_diagnostics.argtypes = [f32p, f32p, f32p, ctypes.c_int64] + [ctypes.c_double] * 5 + [
            ctypes.POINTER(OrSweDiag)]
        L.or_particle_diagnostics.argtypes = [f32p, ctypes.c_int64] + [ctypes.c_double] * 3 + [
            ctypes.POINTER(OrParticleDiag)]
        _LIB = L
    return _LIB


def fp(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(f32p)


def dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(f64p)


def ip(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(i32p)


# ----------------------------------------------------------------------------- java.util.Random

_MULT = 0x5DEECE66D
_MASK = (1 << 48) - 1

_LN2_HI = 6.93147180369123816490e-01
_LN2_LO = 1.90821492927058770002e-10
_TWO54 = 1.80143985094819840000e+16
_LG = (6.666666666666735130e-01, 3.999999999940941908e-01, 2.857142874366239149e-01, 2.222219843214978396e-01,
       1.818357216161805012e-01, 1.531383769920937332e-01, 1.479819860511658591e-01)


def fdlibm_log(x: float) -> float:
    """StrictMath.log: fdlibm's __ieee754_log (Sun's e_log.c), the algorithm java.util.Random's
    nextGaussian calls. Restated from the published fdlibm algorithm for positive finite x."""
    import struct
    bits_ = struct.unpack("<q", struct.pack("<d", x))[0]
    hx = (bits_ >> 32) & 0xFFFFFFFF
    if hx >= 1 << 31:
        hx -= 1 << 32
    lx = bits_ & 0xFFFFFFFF
    k = 0
    if hx < 0x00100000:
        if ((hx & 0x7FFFFFFF) | lx) == 0:
            return -math.inf
        if hx < 0:
            return math.nan
        k -= 54
        x *= _TWO54
        hx = (struct.unpack("<q", struct.pack("<d", x))[0] >> 32) & 0xFFFFFFFF
    if hx >= 0x7FF00000:
        return x + x
    k += (hx >> 20) - 1023
    hx &= 0x000FFFFF
    i = (hx + 0x95F64) & 0x100000
    lo = struct.unpack("<q", struct.pack("<d", x))[0] & 0xFFFFFFFF
    x = struct.unpack("<d", struct.pack("<q", ((hx | (i ^ 0x3FF00000)) << 32) | lo))[0]
    k += i >> 20
    f = x - 1.0
    lg1, lg2, lg3, lg4, lg5, lg6, lg7 = _LG
    if (0x000FFFFF & (2 + hx)) < 3:
        if f == 0.0:
            if k == 0:
                return 0.0
            dk = float(k)
            return dk * _LN2_HI + dk * _LN2_LO
        R = f * f * (0.5 - 0.33333333333333333 * f)
        if k == 0:
            return f - R
        dk = float(k)
        return dk * _LN2_HI - ((R - dk * _LN2_LO) - f)
    s = f / (2.0 + f)
    dk = float(k)
    z = s * s
    i = hx - 0x6147A
    w = z * z
    j = 0x6B851 - hx
    t1 = w * (lg2 + w * (lg4 + w * lg6))
    t2 = z * (lg1 + w * (lg3 + w * (lg5 + w * lg7)))
    i |= j
    R = t2 + t1
    if i > 0:
        hfsq = 0.5 * f * f
        if k == 0:
            return f - (hfsq - s * (hfsq + R))
        return dk * _LN2_HI - ((hfsq - (s * (hfsq + R) + dk * _LN2_LO)) - f)
    if k == 0:
        return f - s * (f - R)
    return dk * _LN2_HI - ((s * (f - R) - dk * _LN2_LO) - f)


class JavaRandom:
    """java.util.Random from its API specification: the 48-bit LCG and its derived draws."""

    def __init__(self, seed: int):
        self.seed = (seed ^ _MULT) & _MASK
        self._next_gaussian = None

    def next(self, bits: int) -> int:
        self.seed = (self.seed * _MULT + 0xB) & _MASK
        r = self.seed >> (48 - bits)
        if r >= 1 << 31:
            r -= 1 << 32
        return r

    def next_int(self, bound: int | None = None) -> int:
        if bound is None:
            return self.next(32)
        if bound & -bound == bound:
            return (bound * self.next(31)) >> 31
        while True:
            bits = self.next(31)
            val = bits % bound
            if ((bits - val + (bound - 1)) & 0xFFFFFFFF) < 1 << 31:
                return val

    def next_float(self) -> np.float32:
        return np.float32(self.next(24)) / np.float32(1 << 24)

    def next_double(self) -> float:
        return ((self.next(26) << 27) + self.next(27)) * (1.0 / (1 << 53))

    def next_gaussian(self) -> float:
        if self._next_gaussian is not None:
            g, self._next_gaussian = self._next_gaussian, None
            return g
        while True:
            v1 = 2 * self.next_double() - 1
            v2 = 2 * self.next_double() - 1
            s = v1 * v1 + v2 * v2
            if 0 < s < 1:
                break
        mult = math.sqrt(-2 * fdlibm_log(s) / s)
        self._next_gaussian = v2 * mult
        return v1 * mult


F = np.float32
WALL = F(1.0)


def flip_column(seed: int, width=8, height=16, ppc=4, rho0=1.0):
    """FlipTest.column (FlipTest.java:134-150): {x, y, m}, ppc jittered particles a cell."""
    r = JavaRandom(seed)
    count = width * height * ppc
    x = np.empty(count, F)
    y = np.empty(count, F)
    m = np.full(count, F(rho0 / ppc), F)
    k = 0
    for row in range(height):
        for col in range(width):
            for _ in range(ppc):
                x[k] = (WALL + F(col)) + r.next_float() * F(0.999)
                y[k] = (WALL + F(row)) + r.next_float() * F(0.999)
                k += 1
    return x, y, m


def slab3(seed: int, n=24, width=6, height=12, ppc=8, rho0=1.0):
    """Flip3Test's slab (Flip3Test.java:307-326): {x, y, z, m} over depth n-3."""
    r = JavaRandom(seed)
    depth = n - 3
    count = width * height * depth * ppc
    x = np.empty(count, F)
    y = np.empty(count, F)
    z = np.empty(count, F)
    m = np.full(count, F(rho0 / ppc), F)
    k = 0
    for layer in range(depth):
        for row in range(height):
            for col in range(width):
                for _ in range(ppc):
                    x[k] = (WALL + F(col)) + r.next_float() * F(0.999)
                    y[k] = (WALL + F(row)) + r.next_float() * F(0.999)
                    z[k] = (WALL + F(layer)) + r.next_float() * F(0.999)
                    k += 1
    return x, y, z, m


def drop3(n=40, radius=8.0, seed=5, ppc=8):
    """Tension3Test's drop (Tension3Test.java:30-62): ppc particles, uniform in each cell whose centre lies within
    ``radius`` of the box's centre, mass 1/ppc. Returns x, y, z, m and the number of cells."""
    centre = n / 2.0
    cells = [(col, row, layer) for layer in range(n) for row in range(n) for col in range(n)
             if math.sqrt((col + 0.5 - centre) ** 2 + (row + 0.5 - centre) ** 2 + (layer + 0.5 - centre) ** 2)
             <= radius]
    count = len(cells) * ppc
    r = JavaRandom(seed)
    at = np.empty((3, count), F)
    k = 0
    for col, row, layer in cells:
        for _ in range(ppc):
            at[0, k] = F(col) + r.next_float() * F(0.999)
            at[1, k] = F(row) + r.next_float() * F(0.999)
            at[2, k] = F(layer) + r.next_float() * F(0.999)
            k += 1
    return at[0], at[1], at[2], np.full(count, F(1.0 / ppc), F), len(cells)


def drop_pressure(make, n=40, radius=8.0, sigma=0.0, sound=200.0):
    """Tension3Test.pressure (Tension3Test.java:30-124) over any 3D step: a drop at rest, no gravity, run for
    0.4 s. ``make(x, y, z, m, params)`` returns an object with ``step()`` and ``read(name)``. Returns the mean
    pressure B(1/J - 1) of the particles in the drop's inner half, averaged over the later steps; 2 sigma / R; R;
    the largest speed of the centre of mass; the fastest particle."""
    bulk = sound * sound
    dt = stable_step(bulk, 1, 20, 0.3)
    steps = math.ceil(0.4 / dt)
    centre = n / 2.0
    x, y, z, m, cells = drop3(n, radius)
    effective = (3 * cells / (4 * math.pi)) ** (1 / 3)
    sim = make(x, y, z, m, (dt, 0.0, 0.0, 0.0, bulk, 1.0, sigma))
    total, samples, fastest, drift = 0.0, 0, 0.0, 0.0
    for s in range(steps):
        sim.step()
        if s >= steps // 3 and s % 5 == 0:
            pos = np.stack([sim.read(a).astype(np.float64) for a in ("x", "y", "z")])
            vel = np.stack([sim.read(a).astype(np.float64) for a in ("u", "v", "w")])
            j = sim.read("j").astype(np.float64)
            fastest = max(fastest, float(np.sqrt((vel ** 2).sum(0)).max()))
            inner = np.sqrt(((pos - centre) ** 2).sum(0)) < 0.5 * effective
            total += float((bulk * (1 / j[inner] - 1)).sum()) / int(inner.sum())
            drift = max(drift, float(np.sqrt((vel.sum(1) ** 2).sum())) / len(x))
            samples += 1
    return total / samples, 2 * sigma / effective, effective, drift, fastest


def relax_box(seed=21, n=48, fill=45, ppc=4):
    """RelaxTest's full box (RelaxTest.java:27-49): fill x fill cells of ppc particles from the wall, mass 1/ppc,
    J = 0.9. Returns x, y, m, j."""
    r = JavaRandom(seed)
    count = fill * fill * ppc
    x, y = np.empty(count, F), np.empty(count, F)
    k = 0
    for row in range(fill):
        for col in range(fill):
            for _ in range(ppc):
                x[k] = (WALL + F(col)) + r.next_float() * F(0.999)
                y[k] = (WALL + F(row)) + r.next_float() * F(0.999)
                k += 1
    return x, y, np.full(count, F(1.0 / ppc), F), np.full(count, F(0.9), F)


def relax_median_j(run, relax):
    """RelaxTest.medianJ (RelaxTest.java:27-65): the box stepped for 0.5 s, sorted every 10 steps, by
    ``run(x, y, m, j, params, steps)``, which returns the particles' J; the median J."""
    bulk = 200.0 ** 2
    dt = stable_step(bulk, 1, 20, 0.3)
    params = flip_params(dt, 0, 0, bulk, 1)
    params[11] = relax
    j = np.sort(run(*relax_box(), params, math.ceil(0.5 / dt)))
    return float(j[len(j) // 2])


def check_laplace(pressure):
    """Tension3Test.aDropsPressureIsTwiceSigmaOverItsRadius's bounds (Tension3Test.java:127-150); ``pressure(radius,
    sigma)`` is drop_pressure over one step implementation."""
    radius = 8.0
    sigma = 0.01 * 200.0 * 200.0 * radius
    none = pressure(radius, 0.0)
    one = pressure(radius, sigma)
    two = pressure(radius, 2 * sigma)
    wide = pressure(1.5 * radius, sigma)
    assert abs(none[0]) < 0.15 * one[1], f"a drop with no tension has pressure {none[0]}"
    ratio = (one[0] - none[0]) / one[1]
    assert 0.3 < ratio < 1.1, f"the pressure is {ratio} of 2 sigma/R"
    doubled = (two[0] - none[0]) / (one[0] - none[0])
    assert 1.6 < doubled < 2.4, f"twice the tension gives {doubled} times the pressure"
    wider = (wide[0] - none[0]) / (one[0] - none[0])
    assert 0.45 < wider < 0.9, f"a drop of 1.5 times the radius has {wider} of the pressure, against 2/3"
    assert one[3] < 0.5, f"the drop's centre of mass moves at {one[3]}"
    return ratio, doubled, wider, one[3]


@dataclass
class Particles:
    """ScatterTest.Particles (ScatterTest.java:453-518): SoA particles in node units."""
    x: np.ndarray
    y: np.ndarray
    u: np.ndarray
    v: np.ndarray
    m: np.ndarray

    def count(self):
        return len(self.x)

    @staticmethod
    def jittered(cells: int, ppc: int, r: JavaRandom) -> "Particles":
        count = cells * cells * ppc
        p = Particles(*(np.empty(count, F) for _ in range(5)))
        k = 0
        for row in range(cells):
            for col in range(cells):
                for _ in range(ppc):
                    p.x[k] = min(F(col) + r.next_float(), np.nextafter(F(col + 1), F(-np.inf)))
                    p.y[k] = min(F(row) + r.next_float(), np.nextafter(F(row + 1), F(-np.inf)))
                    p.u[k] = F(r.next_gaussian())
                    p.v[k] = F(r.next_gaussian())
                    p.m[k] = F(0.5) + r.next_float()
                    k += 1
        return p

    def select(self, order) -> "Particles":
        order = np.asarray(order, dtype=np.int64)
        return Particles(self.x[order].copy(), self.y[order].copy(), self.u[order].copy(), self.v[order].copy(),
                         self.m[order].copy())

    def shuffled(self, r: JavaRandom) -> "Particles":
        order = list(range(self.count()))
        for k in range(len(order) - 1, 0, -1):
            j = r.next_int(k + 1)
            order[k], order[j] = order[j], order[k]
        return self.select(order)

    def sorted_by_cell(self, n: int) -> "Particles":
        keys = cells2(self.x, self.y, n, n)
        return self.select(np.argsort(keys, kind="stable"))

    def where(self, keep) -> "Particles":
        return self.select(np.nonzero(keep)[0])


def cells2(x: np.ndarray, y: np.ndarray, nx: int, ny: int) -> np.ndarray:
    """Scatter.cell for every particle, through the oracle."""
    keys = np.empty(len(x), np.int32)
    lib().or_sort2_keys(fp(x), fp(y), len(x), nx, ny, ip(keys))
    return keys


def bits(a) -> np.ndarray:
    return np.asarray(a, dtype=np.float32).view(np.int32)


def f32_from_bits(b) -> np.ndarray:
    return np.asarray(b, dtype=np.int32).view(np.float32)


def float_bits(v: float) -> int:
    return int(np.array([v], dtype=np.float32).view(np.int32)[0])


# ----------------------------------------------------------------------------- params

def flip_params(dt, gx, gy, bulk, rho0, sigma=0.0) -> np.ndarray:
    """Flip.params (Flip.java:145-211): 28 f32 words; throws on dt <= 0, bulk < 0, rho0 <= 0."""
    if not (dt > 0) or not (bulk >= 0) or not (rho0 > 0):
        raise ValueError(f"dt > 0, bulk >= 0 and rho0 > 0, got dt {dt}, bulk {bulk}, rho0 {rho0}")
    p = np.zeros(28, F)
    p[:6] = [dt, gx, gy, bulk, rho0, sigma]
    return p


def flip3_params(dt, gx, gy, gz, bulk, rho0, sigma=0.0) -> np.ndarray:
    """Flip3.params (Flip3.java:89-103): 7 f32 words."""
    if not (dt > 0) or not (bulk >= 0) or not (rho0 > 0):
        raise ValueError(f"dt > 0, bulk >= 0 and rho0 > 0, got dt {dt}, bulk {bulk}, rho0 {rho0}")
    return np.array([dt, gx, gy, gz, bulk, rho0, sigma], F)


def stable_step(bulk, rho0, speed, courant):
    """Flip.stableStep (Flip.java:214-216)."""
    return courant / (math.sqrt(bulk / rho0) + speed)


def swe_params(g, courant, dx, dy, dry, allow_instability=False) -> np.ndarray:
    """ShallowWater.params (ShallowWater.java:248-271)."""
    if not allow_instability and not (0 < courant <= 0.5):
        raise ValueError(f"a first-order 2D step needs a Courant number in (0, 1/2], got {courant}")
    if not courant > 0:
        raise ValueError(f"a Courant number must be positive, got {courant}")
    return np.array([g, courant, dx, dy, dry], F)


def swe_ticks(seconds: float) -> int:
    """ShallowWater.ticks: seconds to microsecond ticks, rounded (Math.round)."""
    return int(math.floor(seconds * 1_000_000 + 0.5))


def swe_seconds(ticks: int) -> float:
    return ticks / 1_000_000


# ----------------------------------------------------------------------------- oracle state wrappers

class Flip2State:
    """Host arrays of a 2D step, driven through the oracle."""

    FIELDS = ("x", "y", "u", "v", "m", "j", "c00", "c01", "c10", "c11")

    def __init__(self, nx, ny, x, y, m, u=None, v=None, j=None):
        self.nx, self.ny, self.np = nx, ny, len(x)
        self.a = {f: np.zeros(self.np, F) for f in self.FIELDS}
        self.a["x"][:] = x
        self.a["y"][:] = y
        self.a["m"][:] = m
        self.a["j"][:] = 1 if j is None else j
        if u is not None:
            self.a["u"][:] = u
        if v is not None:
            self.a["v"][:] = v
        self.g = {f: np.zeros(nx * ny, F) for f in ("gm", "gmu", "gmv", "gu", "gv")}
        self.s = OrFlip2(nx, ny, self.np, *[fp(self.a[f]) for f in self.FIELDS],
                         *[fp(self.g[f]) for f in ("gm", "gmu", "gmv", "gu", "gv")])

    def step(self, params, physics=(0, 0), relax=False):
        """One FlipStep step; with ``relax``, the step built with relaxation (Flip.advectRelaxing)."""
        step = lib().or_flip2_step_relaxing if relax else lib().or_flip2_step
        step(ctypes.byref(self.s), fp(np.ascontiguousarray(params, F)), OrPhysics(*physics))

    def sort(self):
        cells = (self.nx - 1) * (self.ny - 1)
        starts = np.zeros(cells + 1, np.int32)
        perm = np.zeros(self.np, np.int32)
        tmp = np.zeros(self.np, F)
        lib().or_flip2_sort(ctypes.byref(self.s), ip(starts), ip(perm), fp(tmp))
        return starts


class Flip3State:
    """Host arrays of a 3D step, driven through the oracle."""

    FIELDS = ("x", "y", "z", "u", "v", "w", "m", "j") + tuple(f"c{a}{b}" for a in range(3) for b in range(3))

    def __init__(self, nx, ny, nz, x, y, z, m, **fields):
        self.nx, self.ny, self.nz, self.np = nx, ny, nz, len(x)
        self.a = {f: np.zeros(self.np, F) for f in self.FIELDS}
        self.a["x"][:] = x
        self.a["y"][:] = y
        self.a["z"][:] = z
        self.a["m"][:] = m
        self.a["j"][:] = 1
        for k, v in fields.items():
            self.a[k][:] = v
        nodes = nx * ny * nz
        self.g = {f: np.zeros(nodes, F) for f in ("gm", "gmu", "gmv", "gmw", "gu", "gv", "gw")}
        cs = (f32p * 9)(*[fp(self.a[f"c{a}{b}"]) for a in range(3) for b in range(3)])
        self.s = OrFlip3(nx, ny, nz, self.np, *[fp(self.a[f]) for f in ("x", "y", "z", "u", "v", "w", "m", "j")],
                         cs, *[fp(self.g[f]) for f in ("gm", "gmu", "gmv", "gmw", "gu", "gv", "gw")])

    def step(self, params, physics=(0, 0), tension=False):
        """One Flip3Step step; with ``tension``, the step built with surface tension."""
        p = fp(np.ascontiguousarray(params, F))
        if tension:
            if getattr(self, "_scratch", None) is None:
                self._scratch = np.zeros(8 * self.nx * self.ny * self.nz, F)
            lib().or_flip3_step_tension(ctypes.byref(self.s), p, OrPhysics(*physics), fp(self._scratch))
        else:
            lib().or_flip3_step(ctypes.byref(self.s), p, OrPhysics(*physics))

    def tension_grid(self, params, physics=(0, 0)):
        """The tension's passes and the grid with tension over the grid as it stands (gm..gmw): fills gu, gv, gw
        and returns the last colour and the six stress planes."""
        nodes = self.nx * self.ny * self.nz
        c0, c1 = np.zeros(nodes, F), np.zeros(nodes, F)
        stress = np.zeros(6 * nodes, F)
        pp = np.ascontiguousarray(params, F)
        last = lib().or_tension3_colour(self.nx, self.ny, self.nz, fp(self.g["gm"]), fp(pp), fp(c0), fp(c1))
        colour = c0 if ctypes.addressof(last.contents) == c0.ctypes.data else c1
        lib().or_tension3_stress(self.nx, self.ny, self.nz, fp(colour), fp(stress))
        lib().or_flip3_grid_tension(ctypes.byref(self.s), fp(pp), OrPhysics(*physics), fp(colour), fp(stress))
        return colour, stress.reshape(6, nodes)

    def clear_scatter(self, params, physics=(0, 0)):
        lib().or_flip3_clear(ctypes.byref(self.s))
        lib().or_flip3_scatter(ctypes.byref(self.s), fp(np.ascontiguousarray(params, F)), OrPhysics(*physics))

    def fixed_scatter(self, params, physics=(0, 0)) -> list:
        """The exact scatter (or_fixed_scatter3): m, mu, mv, mw as int64 with 40 fractional bits."""
        nodes = self.nx * self.ny * self.nz
        q = np.zeros(4 * nodes, np.int64)
        lib().or_fixed_scatter3(ctypes.byref(self.s), fp(np.ascontiguousarray(params, F)), OrPhysics(*physics),
                                q.ctypes.data_as(i64p))
        return [q[f * nodes:(f + 1) * nodes] for f in range(4)]

    def sort(self):
        nk = lib().or_key3_count(self.nx, self.ny, self.nz)
        starts = np.zeros(nk + 1, np.int32)
        keys = np.zeros(self.np, np.int32)
        perm = np.zeros(self.np, np.int32)
        tmp = np.zeros(self.np, F)
        lib().or_flip3_sort(ctypes.byref(self.s), ip(starts), ip(keys), ip(perm), fp(tmp))
        return starts, keys, perm


def key3(x, y, z, nx, ny, nz) -> np.ndarray:
    L = lib()
    return np.array([L.or_key3(float(a), float(b), float(c), nx, ny, nz) for a, b, c in zip(x, y, z)], np.int32)


# ----------------------------------------------------------------------------- shallow water


class Clock:
    """The host clock PatchSimulation and Stepper grant budgets from: an i64 tick count.

    The reference's Clock lives in dev.vexelray.sim:vexelray-sim-core (not vendored).
    Its contract, as its call sites use it (PatchSimulation.java:120-145,
    Stepper.java:54-108): grant(end) returns the ticks to end, capped to an i32, and
    holds them outstanding; settle(left) moves the clock by what was spent.
    """

    I32_MAX = 2 ** 31 - 1

    def __init__(self):
        self._now = 0
        self._outstanding = 0

    def now(self):
        return self._now

    def outstanding(self):
        return self._outstanding

    def grant(self, end: int) -> int:
        granted = int(max(0, min(end - self._now, self.I32_MAX)))
        self._outstanding = granted
        return granted

    def settle(self, left: int):
        self._now += self._outstanding - left
        self._outstanding = 0


def slots(k: int):
    """Stepper.slots (Stepper.java:128-130): state in/out, speed in/out/clear, budget in/out."""
    return (k % 2, (k + 1) % 2, k % 3, (k + 1) % 3, (k + 2) % 3, k % 2, (k + 1) % 2)


class OracleSweBackend:
    """The oracle as a Stepper backend: host arrays rotated between dispatches."""

    def __init__(self, nx, ny, edges):
        self.nx, self.ny = nx, ny
        self.edges = np.asarray(edges, np.int32)

    def load(self, h, hu, hv, params, first_speed):
        n = self.nx * self.ny
        self.state = [[np.asarray(h, F).copy(), np.asarray(hu, F).copy(), np.asarray(hv, F).copy()],
                      [np.zeros(n, F), np.zeros(n, F), np.zeros(n, F)]]
        self.speed = [np.array([first_speed], np.int32), np.zeros(1, np.int32), np.zeros(1, np.int32)]
        self.budget = [np.zeros(1, np.int32), np.zeros(1, np.int32)]
        self.clamped_ = np.zeros(1, np.int32)
        self.params = np.asarray(params, F).copy()

    def dispatch(self, k: int):
        si, so, spi, spo, spc, bi, bo = slots(k)
        a, b = self.state[si], self.state[so]
        lib().or_swe_dispatch(self.nx, self.ny, ip(self.edges), fp(self.params), fp(a[0]), fp(a[1]), fp(a[2]),
                              fp(b[0]), fp(b[1]), fp(b[2]), ip(self.speed[spi]), ip(self.speed[spo]),
                              ip(self.speed[spc]), ip(self.budget[bi]), ip(self.budget[bo]), ip(self.clamped_))

    def write_budget(self, slot, ticks):
        self.budget[slot][0] = ticks

    def read_budget(self, slot):
        return int(self.budget[slot][0])

    def read(self, k):
        return [f.copy() for f in self.state[slots(k)[0]]]

    def clamped(self):
        return int(self.clamped_[0])

    def close(self):
        pass


class Stepper:
    """Stepper (Stepper.java:26-130) over a backend: set a state, step it, read it back."""

    def __init__(self, backend, nx, ny):
        self.b = backend
        self.nx, self.ny = nx, ny
        self.dispatched = 0

    def set(self, h, hu, hv, params, end_seconds):
        g = float(np.float32(params[0]))
        dry = float(np.float32(params[4]))
        first = fastest_wave(h, hu, hv, g, dry)
        self.b.load(h, hu, hv, params, first)
        self.dispatched = 0
        self.clock = Clock()
        self.end = swe_ticks(end_seconds)
        self.b.write_budget(0, self.clock.grant(self.end))

    def step(self, steps):
        for _ in range(steps):
            self.b.dispatch(self.dispatched)
            self.dispatched += 1

    def run_until(self, batch, limit):
        while self.ticks() < self.end:
            left = self.b.read_budget(slots(self.dispatched)[5])
            if left == 0:
                self.clock.settle(0)
                self.b.write_budget(slots(self.dispatched)[5], self.clock.grant(self.end))
            if self.dispatched >= limit:
                raise AssertionError(f"the clock is at {self.time()} of {swe_seconds(self.end)} after {limit} steps")
            self.step(batch)

    def ticks(self):
        return self.clock.now() + self.clock.outstanding() - self.b.read_budget(slots(self.dispatched)[5])

    def time(self):
        return swe_seconds(self.ticks())

    def read(self):
        return self.b.read(self.dispatched)

    def clamped(self):
        return self.b.clamped()


def fastest_wave(h, hu, hv, g, dry) -> int:
    h = np.ascontiguousarray(h, F)
    hu = np.ascontiguousarray(hu, F)
    hv = np.ascontiguousarray(hv, F)
    return int(lib().or_swe_fastest_wave(fp(h), fp(hu), fp(hv), len(h), g, dry))


def swe_diagnostics(h, hu, hv, g, dry, dt, dx, dy) -> OrSweDiag:
    d = OrSweDiag()
    h, hu, hv = (np.ascontiguousarray(a, F) for a in (h, hu, hv))
    lib().or_swe_diagnostics(fp(h), fp(hu), fp(hv), len(h), g, dry, dt, dx, dy, ctypes.byref(d))
    return d


def particle_diagnostics(j, speed, sound, dt) -> OrParticleDiag:
    d = OrParticleDiag()
    j = np.ascontiguousarray(j, F)
    lib().or_particle_diagnostics(fp(j), len(j), speed, sound, dt, ctypes.byref(d))
    return d
