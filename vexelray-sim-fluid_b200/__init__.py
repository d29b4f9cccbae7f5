"""vexfluid: the B200 (sm_100a) fluid step of sibarum/vexelray-sim-fluid behind its runner API.

The classes mirror the reference's Java runners, method for method, over the C-ABI library
``libvexfluid.so`` (declared in include/vexfluid.h):

* ``ParticleSimulation``  -- vexelray-sim-fluid-gui/.../gui/ParticleSimulation.java (2D MLS-MPM)
* ``ParticleSimulation3`` -- vexelray-sim-fluid-gui/.../gui/ParticleSimulation3.java (3D MLS-MPM)
* ``PatchSimulation``     -- vexelray-sim-fluid-gui/.../gui/PatchSimulation.java (shallow water)

plus the core's param builders (``Flip.params``, ``Flip3.params``, ``ShallowWater.params``) and the
scatter schedules of ``Scatter``. Errors the reference raises as IllegalArgumentException /
IllegalStateException are raised as ``IllegalArgumentException`` (a ValueError) and
``IllegalStateException`` (a RuntimeError). There is no CPU fallback: without the library or a
CUDA device every call raises.
"""
from __future__ import annotations

import ctypes
import math
import os
import pathlib
import subprocess
from dataclasses import dataclass
from typing import Sequence

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
# the in-tree build; VEXFLUID_LIBRARY names another build of the same library (a variant built for a comparison)
LIBRARY = pathlib.Path(os.environ.get("VEXFLUID_LIBRARY", str(HERE / "libvexfluid.so")))

VF_OK, VF_EINVAL, VF_ESTATE, VF_ENOMEM, VF_ECUDA, VF_ETIMEOUT, VF_ENODEV, VF_EDEVICE = 0, -1, -2, -3, -4, -5, -6, -7
VF_EOS_TAIT = 1
VF_WALL_STICKY_SHIFT = 8
VF_P2G_SHIFT = 16
VF_NO_SORT = 1 << 20
VF_TENSION = 1 << 21
VF_RELAX = 1 << 22
VF_P2G_TILE, VF_P2G_ATOMIC, VF_P2G_WARP, VF_P2G_FIXED, VF_P2G_AUTO = 0, 1, 2, 3, 4
VF_SCATTER_GRID, VF_SCATTER_PRE_REDUCED, VF_SCATTER_GATHER, VF_SCATTER_SEGMENTED = 0, 1, 2, 3
VF3_PASS_SORT, VF3_PASS_CLEAR, VF3_PASS_SCATTER, VF3_PASS_GRID, VF3_PASS_ADVECT = 1, 2, 4, 8, 16
EDGE_WALL, EDGE_OPEN = 0, 1

FIELDS2 = {"x": 0, "y": 1, "u": 2, "v": 3, "m": 4, "j": 5, "c00": 6, "c01": 7, "c10": 8, "c11": 9,
           "gm": 16, "gmu": 17, "gmv": 18, "gu": 19, "gv": 20}
FIELDS3 = {n: k for k, n in enumerate(("x", "y", "z", "u", "v", "w", "m", "j", "c00", "c01", "c02", "c10", "c11",
                                       "c12", "c20", "c21", "c22"))}
FIELDS3.update({"gm": 32, "gmu": 33, "gmv": 34, "gmw": 35, "gu": 36, "gv": 37, "gw": 38})


class VfError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{message} (status {code})")
        self.code = code


class IllegalArgumentException(VfError, ValueError):
    pass


class IllegalStateException(VfError):
    pass


_f32p = ctypes.POINTER(ctypes.c_float)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_vp = ctypes.c_void_p
_LIB = None


def build(quiet: bool = True) -> pathlib.Path:
    """Compiles libvexfluid.so in place (nvcc, sm_100a)."""
    cmd = ["make", "-s" if quiet else "", "-j8", "-C", str(HERE)]
    subprocess.run([c for c in cmd if c], check=True)
    return LIBRARY


class Scene2(ctypes.Structure):
    """vf_scene2: one scene of a batch (grid, particle count, tile shape, Flip.params' first five words)."""
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("particles", ctypes.c_int32),
                ("tile_x", ctypes.c_int32), ("tile_y", ctypes.c_int32), ("params", ctypes.c_int32 * 5)]


BATCH_TILES = ((8, 8), (16, 8), (16, 16), (32, 8), (32, 16))   # VF_BATCH_TILES
BATCH_BLOCKS = (128, 256, 512)                                 # VF_BATCH_BLOCKS


def lib() -> ctypes.CDLL:
    """The loaded library. Raises if it has not been built: there is no fallback."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIBRARY.exists():
        raise RuntimeError(f"libvexfluid.so is not built ({LIBRARY}); run build() first")
    L = ctypes.CDLL(str(LIBRARY))
    sig = {
        "vf_last_error": ([ctypes.c_char_p, ctypes.c_size_t], ctypes.c_int32),
        "vf_version": ([], ctypes.c_int32),
        "vf_device_ok": ([], ctypes.c_int32),
        "vf_binary_version": ([ctypes.POINTER(ctypes.c_int32)], ctypes.c_int32),
        "vf_set_device": ([ctypes.c_int32], ctypes.c_int32),
        "vf_event_create": ([ctypes.POINTER(_vp)], ctypes.c_int32),
        "vf_event_record": ([_vp, _vp], ctypes.c_int32),
        "vf_event_elapsed_ms": ([_vp, _vp, ctypes.POINTER(ctypes.c_float)], ctypes.c_int32),
        "vf_event_destroy": ([_vp], None),
        "vf_host_register": ([_vp, ctypes.c_size_t], ctypes.c_int32),
        "vf_host_unregister": ([_vp], ctypes.c_int32),
        "vf_mpm3_profile": ([_vp, ctypes.c_int32], ctypes.c_int32),
        "vf_mpm3_profile_read": ([_vp, ctypes.c_int32, ctypes.c_char_p, ctypes.c_size_t,
                                  ctypes.POINTER(ctypes.c_double), _i64p], ctypes.c_int32),
        "vf_mpm3_launches": ([_vp], ctypes.c_int64),
        "vf_swe_profile": ([_vp, ctypes.c_int32], ctypes.c_int32),
        "vf_swe_profile_read": ([_vp, ctypes.c_int32, ctypes.c_char_p, ctypes.c_size_t,
                                 ctypes.POINTER(ctypes.c_double), _i64p], ctypes.c_int32),
        "vf_swe_launches": ([_vp], ctypes.c_int64),
        "vf_mpm2_create": ([ctypes.c_int32] * 3 + [ctypes.c_uint32, ctypes.POINTER(_vp)], ctypes.c_int32),
        "vf_mpm2_load": ([_vp] + [_f32p] * 5 + [_i32p, ctypes.c_int32], ctypes.c_int32),
        "vf_mpm2_params": ([_vp, _i32p, ctypes.c_int32], ctypes.c_int32),
        "vf_mpm2_set_graph": ([_vp, ctypes.c_int32], ctypes.c_int32),
        "vf_mpm2_advance": ([_vp, ctypes.c_int32, ctypes.c_int32], ctypes.c_int32),
        "vf_mpm2_step": ([_vp], ctypes.c_int32),
        "vf_mpm2_sort": ([_vp], ctypes.c_int32),
        "vf_mpm2_read": ([_vp, ctypes.c_int32, _f32p, ctypes.c_int64], ctypes.c_int32),
        "vf_mpm2_write": ([_vp, ctypes.c_int32, _f32p, ctypes.c_int64], ctypes.c_int32),
        "vf_mpm2_read_starts": ([_vp, _i32p, ctypes.c_int64], ctypes.c_int32),
        "vf_mpm2_steps": ([_vp], ctypes.c_int64),
        "vf_mpm2_on_gpu": ([_vp], ctypes.c_int32),
        "vf_mpm2_destroy": ([_vp], None),
        "vf_scatter2": ([ctypes.c_int32] * 3 + [_f32p] * 5 + [ctypes.c_int64] + [_f32p] * 3, ctypes.c_int32),
        "vf_fixed_scatter2": ([ctypes.c_int32] * 2 + [_f32p] * 5 + [ctypes.c_int64, ctypes.c_int32, ctypes.c_int32]
                              + [_i32p] * 3, ctypes.c_int32),
        "vf_sort2": ([ctypes.c_int32] * 2 + [_f32p] * 2 + [ctypes.c_int64, _i32p, _i32p], ctypes.c_int32),
        "vf_mpm3_prepare": ([ctypes.c_int32] * 4 + [ctypes.c_uint32, ctypes.POINTER(_vp)], ctypes.c_int32),
        "vf_mpm3_prepare_sparse": ([ctypes.c_int32] * 4 + [ctypes.c_uint32, ctypes.c_int32, ctypes.POINTER(_vp)],
                                   ctypes.c_int32),
        "vf_mpm3_pool_used": ([_vp, _i32p], ctypes.c_int32),
        "vf_mpm3_pool_capacity": ([_vp], ctypes.c_int32),
        "vf_mpm3_set_graph": ([_vp, ctypes.c_int32], ctypes.c_int32),
        "vf_mpm3_schedule": ([_vp], ctypes.c_int32),
        "vf_mpm3_set_fused": ([_vp, ctypes.c_int32], ctypes.c_int32),
        "vf_mpm3_fused": ([_vp], ctypes.c_int32),
        "vf_mpm3_nominal_mass": ([_vp, _f32p], ctypes.c_int32),
        "vf_mpm3_prepared_close": ([_vp], None),
        "vf_mpm3_create": ([_vp, ctypes.POINTER(_vp)], ctypes.c_int32),
        "vf_mpm3_load": ([_vp] + [_f32p] * 7 + [_i32p, ctypes.c_int32], ctypes.c_int32),
        "vf_mpm3_params": ([_vp, _i32p, ctypes.c_int32], ctypes.c_int32),
        "vf_mpm3_advance": ([_vp, ctypes.c_int32], ctypes.c_int32),
        "vf_mpm3_run": ([_vp, ctypes.c_uint32], ctypes.c_int32),
        "vf_mpm3_read": ([_vp, ctypes.c_int32, _f32p, ctypes.c_int64], ctypes.c_int32),
        "vf_mpm3_write": ([_vp, ctypes.c_int32, _f32p, ctypes.c_int64], ctypes.c_int32),
        "vf_mpm3_key_count": ([_vp], ctypes.c_int64),
        "vf_mpm3_read_starts": ([_vp, _i32p, ctypes.c_int64], ctypes.c_int32),
        "vf_mpm3_finish": ([_vp], ctypes.c_int32),
        "vf_mpm3_device_ptr": ([_vp, ctypes.c_char_p, ctypes.POINTER(_vp), _i32p], ctypes.c_int32),
        "vf_mpm3_stream": ([_vp], _vp),
        "vf_mpm3_set_p2g": ([_vp, ctypes.c_int32], ctypes.c_int32),
        "vf_mpm3_read_fixed": ([_vp, ctypes.c_int32, _i64p, ctypes.c_int64], ctypes.c_int32),
        "vf_mpm3_snapshot": ([_vp, _vp, ctypes.c_int64, _i64p], ctypes.c_int32),
        "vf_mpm3_restore": ([_vp, _vp, ctypes.c_int64], ctypes.c_int32),
        "vf_mpm3_touched_nodes": ([_vp, _i64p], ctypes.c_int32),
        "vf_mpm3_steps": ([_vp], ctypes.c_int64),
        "vf_mpm3_on_gpu": ([_vp], ctypes.c_int32),
        "vf_mpm3_destroy": ([_vp], None),
        "vf_mpm3_particle_diagnostics": ([_vp] + [ctypes.c_double] * 3 + [ctypes.POINTER(ctypes.c_double)],
                                         ctypes.c_int32),
        "vf_mpm2_batch_create": ([ctypes.POINTER(Scene2), ctypes.c_int32, ctypes.c_uint32, ctypes.c_int32,
                                  ctypes.POINTER(_vp)], ctypes.c_int32),
        "vf_mpm2_batch_load": ([_vp] + [_f32p] * 5, ctypes.c_int32),
        "vf_mpm2_batch_advance": ([_vp, ctypes.c_int32], ctypes.c_int32),
        "vf_mpm2_batch_finish": ([_vp], ctypes.c_int32),
        "vf_mpm2_batch_set_wait_limit": ([_vp, ctypes.c_int32], ctypes.c_int32),
        "vf_mpm2_batch_read": ([_vp, ctypes.c_int32, ctypes.c_int32, _f32p, ctypes.c_int64], ctypes.c_int32),
        "vf_mpm2_batch_config": ([_vp, ctypes.c_int32] + [_i32p] * 4, ctypes.c_int32),
        "vf_mpm2_batch_phases": ([_vp, ctypes.POINTER(ctypes.c_double), _i64p], ctypes.c_int32),
        "vf_mpm2_batch_particles": ([_vp], ctypes.c_int64),
        "vf_mpm2_batch_steps": ([_vp], ctypes.c_int64),
        "vf_mpm2_batch_launches": ([_vp], ctypes.c_int64),
        "vf_mpm2_batch_stream": ([_vp], _vp),
        "vf_mpm2_batch_destroy": ([_vp], None),
        "vf_mpm2_autotune": ([ctypes.POINTER(Scene2), ctypes.c_int32, ctypes.c_uint32] + [_f32p] * 5 +
                             [ctypes.c_char_p, _i32p, _i32p], ctypes.c_int32),
        "vf_swe_state": ([_vp] + [ctypes.POINTER(_vp)] * 3, ctypes.c_int32),
        "vf_swe_measure_speed": ([_vp], ctypes.c_int32),
        "vf_swe_restrict": ([_vp, _vp], ctypes.c_int32),
        "vf_swe_prolong": ([_vp, ctypes.c_int32, ctypes.c_int32, _vp], ctypes.c_int32),
        "vf_swe_restrict_patch": ([_vp, ctypes.c_int32, ctypes.c_int32, _vp] + [ctypes.c_int32] * 4, ctypes.c_int32),
        "vf_swe_copy_state": ([_vp, _vp], ctypes.c_int32),
        "vf_swe_jump_indicator": ([_vp, ctypes.c_int32, _f32p, ctypes.c_int32], ctypes.c_int32),
        "vf_cnn_param_count": ([], ctypes.c_int64),
        "vf_cnn_create": ([ctypes.c_int32] * 4 + [ctypes.c_float, ctypes.c_float, ctypes.POINTER(_vp)], ctypes.c_int32),
        "vf_cnn_params": ([_vp, _f32p, ctypes.c_int64, ctypes.c_int32], ctypes.c_int32),
        "vf_cnn_put": ([_vp, ctypes.c_int32, ctypes.c_int32, _vp, _vp, _vp, ctypes.c_int32], ctypes.c_int32),
        "vf_cnn_loss": ([_vp, _i32p, ctypes.c_int32, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)],
                        ctypes.c_int32),
        "vf_cnn_gradients": ([_vp, _i32p, ctypes.c_int32, _f32p, ctypes.POINTER(ctypes.c_double)], ctypes.c_int32),
        "vf_cnn_train": ([_vp, _i32p, ctypes.c_int32, ctypes.c_float, ctypes.POINTER(ctypes.c_double)], ctypes.c_int32),
        "vf_cnn_correct": ([_vp] * 5, ctypes.c_int32),
        "vf_cnn_predict": ([_vp] * 5, ctypes.c_int32),
        "vf_cnn_apply": ([_vp] * 5, ctypes.c_int32),
        "vf_cnn_fluxes": ([_vp, ctypes.c_int32, _f32p], ctypes.c_int32),
        "vf_cnn_stream": ([_vp], _vp),
        "vf_cnn_set_path": ([_vp, ctypes.c_int32], ctypes.c_int32),
        "vf_cnn_status": ([_vp], ctypes.c_int32),
        "vf_cnn_profile": ([_vp, ctypes.c_int32], ctypes.c_int32),
        "vf_cnn_profile_read": ([_vp, ctypes.c_int32, ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_double),
                                 _i64p], ctypes.c_int32),
        "vf_cnn_launches": ([_vp], ctypes.c_int64),
        "vf_cnn_destroy": ([_vp], None),
        "vf_swe_learned_create": ([ctypes.c_int32, ctypes.c_int32, _vp, ctypes.c_int64, ctypes.c_int32,
                                   ctypes.c_int32, ctypes.c_float, ctypes.c_int32, ctypes.c_float,
                                   ctypes.POINTER(_vp)],
                                  ctypes.c_int32),
        "vf_swe_learned_load": ([_vp, _f32p, _f32p, _f32p], ctypes.c_int32),
        "vf_swe_learned_advance": ([_vp, ctypes.c_int64], ctypes.c_int32),
        "vf_swe_learned_read": ([_vp, _f32p, _f32p, _f32p], ctypes.c_int32),
        "vf_swe_learned_counts": ([_vp, ctypes.POINTER(ctypes.c_int64)], ctypes.c_int32),
        "vf_swe_learned_coarse": ([_vp], _vp),
        "vf_swe_learned_destroy": ([_vp], None),
        "vf_swe_create": ([ctypes.c_int32, ctypes.c_int32, _i32p, ctypes.POINTER(_vp)], ctypes.c_int32),
        "vf_swe_load": ([_vp] + [_f32p] * 3 + [_i32p, ctypes.c_int32], ctypes.c_int32),
        "vf_swe_params": ([_vp, _i32p, ctypes.c_int32], ctypes.c_int32),
        "vf_swe_advance": ([_vp, ctypes.c_int64, ctypes.c_int32, _i32p, _i64p, _i64p], ctypes.c_int32),
        "vf_swe_read": ([_vp] + [_f32p] * 3, ctypes.c_int32),
        "vf_swe_fastest_wave": ([_vp, ctypes.POINTER(ctypes.c_double)], ctypes.c_int32),
        "vf_swe_clamped": ([_vp, _i32p], ctypes.c_int32),
        "vf_swe_now": ([_vp], ctypes.c_int64),
        "vf_swe_steps": ([_vp], ctypes.c_int64),
        "vf_swe_dispatch": ([_vp, ctypes.c_int32], ctypes.c_int32),
        "vf_swe_dispatched": ([_vp], ctypes.c_int64),
        "vf_swe_set_tile_width": ([_vp, ctypes.c_int32], ctypes.c_int32),
        "vf_swe_tile_width": ([_vp], ctypes.c_int32),
        "vf_swe_set_overlap": ([_vp, ctypes.c_int32], ctypes.c_int32),
        "vf_swe_set_exact": ([_vp, ctypes.c_int32], ctypes.c_int32),
        "vf_swe_exact": ([_vp], ctypes.c_int32),
        "vf_swe_snapshot": ([_vp, _vp, ctypes.c_int64, _i64p], ctypes.c_int32),
        "vf_swe_restore": ([_vp, _vp, ctypes.c_int64], ctypes.c_int32),
        "vf_swe_write_budget": ([_vp, ctypes.c_int32, ctypes.c_int32], ctypes.c_int32),
        "vf_swe_read_budget": ([_vp, ctypes.c_int32, _i32p], ctypes.c_int32),
        "vf_swe_diagnostics": ([_vp] + [ctypes.c_double] * 5 + [ctypes.POINTER(ctypes.c_double)], ctypes.c_int32),
        "vf_swe_stream": ([_vp], _vp),
        "vf_swe_on_gpu": ([_vp], ctypes.c_int32),
        "vf_swe_destroy": ([_vp], None),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _LIB = L
    return L


def last_error() -> str:
    buf = ctypes.create_string_buffer(1024)
    lib().vf_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(code: int) -> None:
    if code == VF_OK:
        return
    msg = last_error()
    if code == VF_EINVAL:
        raise IllegalArgumentException(code, msg)
    if code == VF_ESTATE:
        raise IllegalStateException(code, msg)
    raise VfError(code, msg)


def _snapshot(fn, h) -> bytes:
    size = ctypes.c_int64()
    check(fn(h, None, 0, ctypes.byref(size)))
    buf = ctypes.create_string_buffer(size.value)
    check(fn(h, buf, size.value, ctypes.byref(size)))
    return buf.raw[: size.value]


def _f32(a, n=None) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32)
    if n is not None and a.shape != (n,):
        raise IllegalArgumentException(VF_EINVAL, f"expected {n} values, got shape {a.shape}")
    return a


def _fp(a: np.ndarray):
    return a.ctypes.data_as(_f32p)


def _ip(a: np.ndarray):
    return a.ctypes.data_as(_i32p)


def _words(params) -> np.ndarray:
    p = np.asarray(params)
    if p.dtype == np.float32:
        return np.ascontiguousarray(p.view(np.int32))
    return np.ascontiguousarray(p, dtype=np.int32)


def _bits(v: float) -> int:
    return int(np.array([v], dtype=np.float32).view(np.int32)[0])


def _profile_read(fn, h):
    """{kernel name: (total ms, launches)} from a handle's profiler."""
    out = {}
    k = 0
    buf = ctypes.create_string_buffer(128)
    while True:
        ms = ctypes.c_double()
        n = ctypes.c_int64()
        if fn(h, k, buf, len(buf), ctypes.byref(ms), ctypes.byref(n)) != VF_OK:
            break
        out[buf.value.decode()] = (ms.value, n.value)
        k += 1
    return out


class Event:
    """A CUDA event, recorded on a handle's stream."""

    def __init__(self):
        e = _vp()
        check(lib().vf_event_create(ctypes.byref(e)))
        self._e = e

    def record(self, stream) -> None:
        check(lib().vf_event_record(self._e, stream))

    def elapsed_ms(self, stop: "Event") -> float:
        ms = ctypes.c_float()
        check(lib().vf_event_elapsed_ms(self._e, stop._e, ctypes.byref(ms)))
        return ms.value

    def __del__(self):
        try:
            lib().vf_event_destroy(self._e)
        except Exception:
            pass


def set_device(device: int) -> None:
    check(lib().vf_set_device(device))


class Pinned:
    """Pins numpy arrays' host memory for the duration of a with-block (cudaHostRegister)."""

    def __init__(self, *arrays):
        self.arrays = [a for a in arrays if a.nbytes]

    def __enter__(self):
        for a in self.arrays:
            check(lib().vf_host_register(a.ctypes.data, a.nbytes))
        return self

    def __exit__(self, *exc):
        for a in self.arrays:
            lib().vf_host_unregister(a.ctypes.data)


# ------------------------------------------------------------------------------------- params

def flip_params(dt, gx, gy, bulk, rho0, sigma=0.0, relax=0.0) -> np.ndarray:
    """Flip.params (Flip.java:145-211): 28 words of f32 bits; ``relax`` is word 11 (Flip.RELAX), the rate at
    which a step built with relaxation draws J toward the volume the mass gives."""
    if not (dt > 0) or not (bulk >= 0) or not (rho0 > 0):
        raise IllegalArgumentException(VF_EINVAL, f"dt > 0, bulk >= 0 and rho0 > 0, got dt {dt}, bulk {bulk}, "
                                                  f"rho0 {rho0}")
    w = np.zeros(28, np.int32)
    for k, v in enumerate((dt, gx, gy, bulk, rho0, sigma)):
        w[k] = _bits(v)
    w[11] = _bits(relax)
    return w


def flip3_params(dt, gx, gy, gz, bulk, rho0, sigma=0.0) -> np.ndarray:
    """Flip3.params (Flip3.java:89-103): 7 words of f32 bits."""
    if not (dt > 0) or not (bulk >= 0) or not (rho0 > 0):
        raise IllegalArgumentException(VF_EINVAL, f"dt > 0, bulk >= 0 and rho0 > 0, got dt {dt}, bulk {bulk}, "
                                                  f"rho0 {rho0}")
    return np.array([_bits(v) for v in (dt, gx, gy, gz, bulk, rho0, sigma)], np.int32)


def stable_step(bulk, rho0, speed, courant) -> float:
    """Flip.stableStep (Flip.java:214-216)."""
    return courant / (math.sqrt(bulk / rho0) + speed)


def swe_params(g, courant, dx, dy, dry=1e-6, allow_instability=False) -> np.ndarray:
    """ShallowWater.params / paramsAllowingInstability (ShallowWater.java:248-271)."""
    if not allow_instability and not (0 < courant <= 0.5):
        raise IllegalArgumentException(VF_EINVAL, "a first-order 2D step needs a Courant number in (0, 1/2], got "
                                       + str(courant))
    if not courant > 0:
        raise IllegalArgumentException(VF_EINVAL, f"a Courant number must be positive, got {courant}")
    return np.array([_bits(v) for v in (g, courant, dx, dy, dry)], np.int32)


TICKS_PER_SECOND = 1_000_000


def ticks(seconds: float) -> int:
    """ShallowWater.ticks: seconds to microsecond ticks, Math.round."""
    return int(math.floor(seconds * TICKS_PER_SECOND + 0.5))


def seconds(t: int) -> float:
    return t / TICKS_PER_SECOND


# ------------------------------------------------------------------------------------- 2D

class ParticleSimulation:
    """ParticleSimulation (ParticleSimulation.java): a 2D particle fluid in one walled box on the GPU."""

    def __init__(self, nx: int, ny: int, particles: int, *, tait: bool = False, sticky: int = 0, relax: bool = False):
        L = lib()
        h = _vp()
        flags = (VF_EOS_TAIT if tait else 0) | (int(sticky) << VF_WALL_STICKY_SHIFT) | (VF_RELAX if relax else 0)
        check(L.vf_mpm2_create(nx, ny, particles, flags, ctypes.byref(h)))
        self._h = h
        self._nx, self._ny, self._np = nx, ny, particles

    def nx(self):
        return self._nx

    def ny(self):
        return self._ny

    def particles(self):
        return self._np

    def on_gpu(self) -> bool:
        return bool(lib().vf_mpm2_on_gpu(self._h))

    def load(self, x, y, u, v, m, params) -> None:
        n = self._np
        a = [_f32(q, n) for q in (x, y, u, v, m)]
        w = _words(params)
        check(lib().vf_mpm2_load(self._h, *[_fp(q) for q in a], _ip(w), len(w)))

    def params(self, params) -> None:
        w = _words(params)
        check(lib().vf_mpm2_params(self._h, _ip(w), len(w)))

    def advance(self, count: int, sort_every: int) -> None:
        check(lib().vf_mpm2_advance(self._h, count, sort_every))

    def set_graph(self, on: bool) -> None:
        """advance() replays a sort and the sort_every steps after it from one captured CUDA graph (off by default)."""
        check(lib().vf_mpm2_set_graph(self._h, 1 if on else 0))

    def step(self) -> None:
        """One FlipStep.step() without counting it (the test Rig's run(step.step()))."""
        check(lib().vf_mpm2_step(self._h))

    def sort(self) -> None:
        """One FlipStep.sort() (the test Rig's run(step.sort()))."""
        check(lib().vf_mpm2_sort(self._h))

    def read(self, name: str) -> np.ndarray:
        f = FIELDS2[name]
        n = self._nx * self._ny if f >= 16 else self._np
        out = np.empty(n, np.float32)
        check(lib().vf_mpm2_read(self._h, f, _fp(out), n))
        return out

    def write(self, name: str, values) -> None:
        a = _f32(values, self._np)
        check(lib().vf_mpm2_write(self._h, FIELDS2[name], _fp(a), self._np))

    def grid(self):
        return [self.read("gm"), self.read("gmu"), self.read("gmv")]

    def masses(self):
        return self.read("m")

    def velocities(self):
        return [self.read("u"), self.read("v")]

    def positions(self):
        return [self.read("x"), self.read("y")]

    def compression(self, j=None):
        if j is None:
            return self.read("j")
        self.write("j", j)

    def starts(self) -> np.ndarray:
        out = np.empty((self._nx - 1) * (self._ny - 1) + 1, np.int32)
        check(lib().vf_mpm2_read_starts(self._h, _ip(out), len(out)))
        return out

    def steps(self) -> int:
        return int(lib().vf_mpm2_steps(self._h))

    def close(self) -> None:
        if self._h:
            lib().vf_mpm2_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class Scene:
    """One scene of a batch: an nx x ny grid, its particles' count, the Flip.params words it steps with
    (the first five are used) and its tile shape (None: the default, or the tuner's choice)."""
    nx: int
    ny: int
    particles: int
    params: Sequence[int]
    tile: tuple | None = None

    def _c(self) -> Scene2:
        w = _words(self.params)
        if len(w) < 5:
            raise IllegalArgumentException(VF_EINVAL, f"Flip.params has at least 5 words, got {len(w)}")
        tx, ty = self.tile or (0, 0)
        return Scene2(self.nx, self.ny, self.particles, tx, ty, (ctypes.c_int32 * 5)(*[int(v) for v in w[:5]]))


def _scene_table(scenes: Sequence[Scene]):
    return (Scene2 * len(scenes))(*[s._c() for s in scenes])


def _concat(scenes, arrays, name):
    total = sum(s.particles for s in scenes)
    a = np.ascontiguousarray(np.concatenate([np.asarray(q, np.float32).ravel() for q in arrays])
                             if isinstance(arrays, (list, tuple)) else np.asarray(arrays, np.float32).ravel())
    if a.size != total:
        raise IllegalArgumentException(VF_EINVAL, f"{name} holds {a.size} floats for {total} particles")
    return a


class BatchSimulation:
    """Many independent 2D scenes stepped together: one cooperative persistent kernel launch per step over
    every scene, replayed from CUDA graphs (vf_mpm2_batch_*). Particle arrays are the scenes' particles one
    scene after another (or a list of per-scene arrays)."""

    def __init__(self, scenes: Sequence[Scene], *, tait: bool = False, sticky: int = 0, block: int = 0):
        self._scenes = list(scenes)
        self._flags = (VF_EOS_TAIT if tait else 0) | (int(sticky) << VF_WALL_STICKY_SHIFT)
        h = _vp()
        check(lib().vf_mpm2_batch_create(_scene_table(self._scenes), len(self._scenes), self._flags, block,
                                         ctypes.byref(h)))
        self._h = h

    def load(self, x, y, u, v, m) -> None:
        a = [_concat(self._scenes, q, n) for q, n in ((x, "x"), (y, "y"), (u, "u"), (v, "v"), (m, "m"))]
        check(lib().vf_mpm2_batch_load(self._h, *[_fp(q) for q in a]))

    def advance(self, count: int) -> None:
        check(lib().vf_mpm2_batch_advance(self._h, count))

    def finish(self) -> None:
        check(lib().vf_mpm2_batch_finish(self._h))

    def set_wait_limit(self, polls: int) -> None:
        """Polls a CTA makes at a grid barrier before it gives up (0: the default, about a second). A load restores
        the default."""
        check(lib().vf_mpm2_batch_set_wait_limit(self._h, polls))

    def read(self, scene: int, name: str) -> np.ndarray:
        f = FIELDS2[name]
        sc = self._scenes[scene]
        n = sc.nx * sc.ny if f >= 16 else sc.particles
        out = np.empty(n, np.float32)
        check(lib().vf_mpm2_batch_read(self._h, scene, f, _fp(out), n))
        return out

    def config(self, scene: int = 0) -> dict:
        v = [np.zeros(1, np.int32) for _ in range(4)]
        check(lib().vf_mpm2_batch_config(self._h, scene, *[_ip(q) for q in v]))
        return {"tile": (int(v[0][0]), int(v[1][0])), "block": int(v[2][0]), "ctas": int(v[3][0])}

    PHASES = ("tile_scan", "cell_scan", "permute", "scatter", "gather")

    def phases(self) -> dict:
        """Device ms of each phase of the step summed over the launches since the last call, and the launches."""
        ms = (ctypes.c_double * 5)()
        n = np.zeros(1, np.int64)
        check(lib().vf_mpm2_batch_phases(self._h, ms, n.ctypes.data_as(_i64p)))
        out = {k: ms[i] for i, k in enumerate(self.PHASES)}
        out["launches"] = int(n[0])
        return out

    def particles(self) -> int:
        return int(lib().vf_mpm2_batch_particles(self._h))

    def steps(self) -> int:
        return int(lib().vf_mpm2_batch_steps(self._h))

    def launches(self) -> int:
        return int(lib().vf_mpm2_batch_launches(self._h))

    def stream(self):
        return lib().vf_mpm2_batch_stream(self._h)

    def close(self) -> None:
        if self._h:
            lib().vf_mpm2_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(scenes: Sequence[Scene], x, y, u, v, m, *, tait: bool = False, sticky: int = 0,
             cache: str | os.PathLike | None = None):
    """vf_mpm2_autotune: picks each scene's tile shape and the batch's block size, timing what the JSON cache
    does not hold. Returns (scenes with their tiles set, block, trials timed)."""
    table = _scene_table(scenes)
    a = [_concat(scenes, q, n) for q, n in ((x, "x"), (y, "y"), (u, "u"), (v, "v"), (m, "m"))]
    block = np.zeros(1, np.int32)
    trials = np.zeros(1, np.int32)
    flags = (VF_EOS_TAIT if tait else 0) | (int(sticky) << VF_WALL_STICKY_SHIFT)
    path = None if cache is None else os.fsencode(os.fspath(cache))
    check(lib().vf_mpm2_autotune(table, len(scenes), flags, *[_fp(q) for q in a], path, _ip(block), _ip(trials)))
    tuned = [Scene(s.nx, s.ny, s.particles, s.params, (int(table[k].tile_x), int(table[k].tile_y)))
             for k, s in enumerate(scenes)]
    return tuned, int(block[0]), int(trials[0])


class FluxNet:
    """The flux-correction network of the learned coarse shallow-water solver (vf_cnn_*): a 3-layer 5x5 CNN
    (3 -> 32 -> 32 -> 6) whose output's divergence corrects a coarse state, trained with Adam on samples
    (S, P, T) held on the device (see vexfluid.h for the loss)."""

    def __init__(self, nx: int, ny: int, *, batch: int = 1, samples: int = 1, s_flux: float = 1e-3,
                 s_res: float = 1e-3):
        h = _vp()
        check(lib().vf_cnn_create(nx, ny, batch, samples, s_flux, s_res, ctypes.byref(h)))
        self._h = h
        self.nx, self.ny, self.s_flux, self.s_res = nx, ny, s_flux, s_res
        self.batch, self.samples = batch, samples

    @staticmethod
    def count() -> int:
        return int(lib().vf_cnn_param_count())

    def params(self, values=None) -> np.ndarray | None:
        n = self.count()
        if values is None:
            out = np.empty(n, np.float32)
            check(lib().vf_cnn_params(self._h, _fp(out), n, 0))
            return out
        a = _f32(values, n)
        check(lib().vf_cnn_params(self._h, _fp(a), n, 1))
        return None

    def put(self, slot: int, kind: int, h, hu, hv) -> None:
        """Sample slot's part kind (0 S, 1 P, 2 T) from host arrays."""
        n = self.nx * self.ny
        a = [_f32(np.asarray(q).ravel(), n) for q in (h, hu, hv)]
        check(lib().vf_cnn_put(self._h, slot, kind, *[q.ctypes.data_as(_vp) for q in a], 1))

    def put_state(self, slot: int, kind: int, sim: "PatchSimulation") -> None:
        """Sample slot's part kind from a PatchSimulation's current device state (same grid)."""
        ptr = sim.device_state()
        check(lib().vf_cnn_put(self._h, slot, kind, *ptr, 0))

    def _slots(self, slots):
        a = np.ascontiguousarray(np.atleast_1d(slots), np.int32)
        return _ip(a), len(a), a

    def loss(self, slots) -> tuple[float, float]:
        p, n, keep = self._slots(slots)
        l, lp = ctypes.c_double(), ctypes.c_double()
        check(lib().vf_cnn_loss(self._h, p, n, ctypes.byref(l), ctypes.byref(lp)))
        return l.value, lp.value

    def gradients(self, slots) -> tuple[np.ndarray, float]:
        p, n, keep = self._slots(slots)
        g = np.empty(self.count(), np.float32)
        l = ctypes.c_double()
        check(lib().vf_cnn_gradients(self._h, p, n, _fp(g), ctypes.byref(l)))
        return g, l.value

    def train(self, slots, lr: float) -> float:
        p, n, keep = self._slots(slots)
        l = ctypes.c_double()
        check(lib().vf_cnn_train(self._h, p, n, lr, ctypes.byref(l)))
        return l.value

    def fluxes(self, slot: int = 0) -> np.ndarray:
        out = np.empty(self.nx * self.ny * 8, np.float32)
        check(lib().vf_cnn_fluxes(self._h, slot, _fp(out)))
        return out.reshape(self.ny, self.nx, 8)

    def correct(self, sim: "PatchSimulation") -> None:
        """The correction predicted from a PatchSimulation's current state and applied to it in place, and its
        wave speed measured again."""
        check(lib().vf_cnn_correct(self._h, *sim.device_state(), sim.stream()))
        check(lib().vf_swe_measure_speed(sim._h))

    def predict(self, sim: "PatchSimulation") -> None:
        """The correction predicted from the current state (an interval's start)."""
        check(lib().vf_cnn_predict(self._h, *sim.device_state(), sim.stream()))

    def apply(self, sim: "PatchSimulation") -> None:
        """The last prediction applied to the current state (the interval's end), its wave speed measured again."""
        check(lib().vf_cnn_apply(self._h, *sim.device_state(), sim.stream()))
        check(lib().vf_swe_measure_speed(sim._h))

    def set_path(self, path: int) -> None:
        """The convolutions' kernels: 0 tcgen05 for the 32-channel inputs (default), 1 mma.sync row-blocked, 2
        mma.sync one output row per warp."""
        check(lib().vf_cnn_set_path(self._h, path))

    def status(self) -> None:
        check(lib().vf_cnn_status(self._h))

    def profile(self, on: bool) -> None:
        check(lib().vf_cnn_profile(self._h, 1 if on else 0))

    def profile_read(self) -> dict:
        return _profile_read(lib().vf_cnn_profile_read, self._h)

    def launches(self) -> int:
        return int(lib().vf_cnn_launches(self._h))

    def stream(self):
        return lib().vf_cnn_stream(self._h)

    def close(self) -> None:
        if self._h:
            lib().vf_cnn_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def scatter2(mode: int, nx: int, ny: int, x, y, u, v, m):
    """One bilinear P2G (Scatter.kernel / preReduced / gather / segmented) of host particles."""
    n = len(x)
    a = [_f32(q, n) for q in (x, y, u, v, m)]
    out = [np.zeros(nx * ny, np.float32) for _ in range(3)]
    check(lib().vf_scatter2(mode, nx, ny, *[_fp(q) for q in a], n, *[_fp(o) for o in out]))
    return out


def fixed_scatter2(nx: int, ny: int, x, y, u, v, m, mass_bits: int, velocity_bits: int):
    """FixedScatter.kernel: the bilinear P2G in wrapping i32 quanta."""
    n = len(x)
    a = [_f32(q, n) for q in (x, y, u, v, m)]
    out = [np.zeros(nx * ny, np.int32) for _ in range(3)]
    check(lib().vf_fixed_scatter2(nx, ny, *[_fp(q) for q in a], n, mass_bits, velocity_bits,
                                  *[_ip(o) for o in out]))
    return out


def sort2(nx: int, ny: int, x, y):
    """The device's stable sort by Scatter.cell: (perm, starts)."""
    n = len(x)
    xs, ys = _f32(x, n), _f32(y, n)
    perm = np.empty(n, np.int32)
    starts = np.empty((nx - 1) * (ny - 1) + 1, np.int32)
    check(lib().vf_sort2(nx, ny, _fp(xs), _fp(ys), n, _ip(perm), _ip(starts)))
    return perm, starts


# ------------------------------------------------------------------------------------- 3D

class Prepared:
    """ParticleSimulation3.Prepared (ParticleSimulation3.java:51-103)."""

    def __init__(self, handle, nx, ny, nz, particles):
        self._p = handle
        self.nx, self.ny, self.nz, self.particles = nx, ny, nz, particles

    def close(self):
        if self._p:
            lib().vf_mpm3_prepared_close(self._p)
            self._p = None


class ParticleSimulation3:
    """ParticleSimulation3 (ParticleSimulation3.java): a 3D particle fluid in one walled box on the GPU.

    ``schedule`` is the scatter: VF_P2G_TILE (default; sorts every step), VF_P2G_ATOMIC, VF_P2G_WARP, VF_P2G_FIXED
    (exact: 64-bit fixed-point sums, the same grid in any order) or VF_P2G_AUTO (the fastest for the size: the
    warp-aggregated scatter for scenes of the reference's scale, the tile for large ones).
    ``sort=False`` keeps the particles in load order, as the reference's Flip3Step does.
    ``tension=True`` adds surface tension's passes (ParticleSimulation3(..., tension)); its strength is sigma, the
    seventh params word (``flip3_params(..., sigma)``).
    ``pool_bricks=N`` stores the grid sparsely, in a pool of N bricks of 8^3 nodes through a page table over the
    domain (the tiled schedule only, without tension); ``pool_used()`` is what the last step took.
    """

    @staticmethod
    def prepare(nx, ny, nz, particles, *, tait=False, sticky=0, schedule=VF_P2G_TILE, sort=True,
                tension=False, pool_bricks=None) -> Prepared:
        flags = ((VF_EOS_TAIT if tait else 0) | (int(sticky) << VF_WALL_STICKY_SHIFT) | (schedule << VF_P2G_SHIFT)
                 | (0 if sort else VF_NO_SORT) | (VF_TENSION if tension else 0))
        p = _vp()
        if pool_bricks is None:
            check(lib().vf_mpm3_prepare(nx, ny, nz, particles, flags, ctypes.byref(p)))
        else:
            check(lib().vf_mpm3_prepare_sparse(nx, ny, nz, particles, flags, int(pool_bricks), ctypes.byref(p)))
        return Prepared(p, nx, ny, nz, particles)

    def __init__(self, nx_or_prepared, ny=None, nz=None, particles=None, **kw):
        prepared = nx_or_prepared if isinstance(nx_or_prepared, Prepared) else \
            ParticleSimulation3.prepare(nx_or_prepared, ny, nz, particles, **kw)
        h = _vp()
        if not prepared._p:
            raise IllegalStateException(VF_ESTATE, "this preparation has already been made a simulation, or closed")
        check(lib().vf_mpm3_create(prepared._p, ctypes.byref(h)))
        prepared._p = None
        self._h = h
        self._nx, self._ny, self._nz, self._np = prepared.nx, prepared.ny, prepared.nz, prepared.particles

    def nx(self):
        return self._nx

    def ny(self):
        return self._ny

    def nz(self):
        return self._nz

    def particles(self):
        return self._np

    def on_gpu(self) -> bool:
        return bool(lib().vf_mpm3_on_gpu(self._h))

    def load(self, at, velocity, mass, params) -> None:
        n = self._np
        a = [_f32(q, n) for q in (at[0], at[1], at[2], velocity[0], velocity[1], velocity[2], mass)]
        w = _words(params)
        check(lib().vf_mpm3_load(self._h, *[_fp(q) for q in a], _ip(w), len(w)))

    def params(self, params) -> None:
        w = _words(params)
        check(lib().vf_mpm3_params(self._h, _ip(w), len(w)))

    def advance(self, count: int) -> None:
        check(lib().vf_mpm3_advance(self._h, count))

    def run(self, passes: int) -> None:
        """Passes of one step (VF3_PASS_*), as the test Rig runs a sub-list of Flip3Step.step()."""
        check(lib().vf_mpm3_run(self._h, passes))

    def read(self, name: str) -> np.ndarray:
        f = FIELDS3[name]
        n = self._nx * self._ny * self._nz if f >= 32 else self._np
        out = np.empty(n, np.float32)
        check(lib().vf_mpm3_read(self._h, f, _fp(out), n))
        return out

    def write(self, name: str, values) -> None:
        a = _f32(values, self._np)
        check(lib().vf_mpm3_write(self._h, FIELDS3[name], _fp(a), self._np))

    def grid(self):
        return [self.read("gm"), self.read("gmu"), self.read("gmv"), self.read("gmw")]

    def velocities(self):
        return [self.read("u"), self.read("v"), self.read("w")]

    def positions(self):
        return [self.read("x"), self.read("y"), self.read("z")]

    def compression(self):
        """ParticleSimulation3.compression (ParticleSimulation3.java:312-333): J of the particles holding at least
        half the smallest loaded mass."""
        j = self.read("j")
        m = self.read("m")
        nominal = np.empty(1, np.float32)
        check(lib().vf_mpm3_nominal_mass(self._h, _fp(nominal)))
        keep = m >= np.float32(0.5) * nominal[0]
        return j if keep.all() else j[keep]

    def key_count(self) -> int:
        return int(lib().vf_mpm3_key_count(self._h))

    def starts(self) -> np.ndarray:
        out = np.empty(self.key_count() + 1, np.int32)
        check(lib().vf_mpm3_read_starts(self._h, _ip(out), len(out)))
        return out

    def finish(self) -> None:
        check(lib().vf_mpm3_finish(self._h))

    def device_ptr(self, name: str):
        p = _vp()
        stride = ctypes.c_int32()
        check(lib().vf_mpm3_device_ptr(self._h, name.encode(), ctypes.byref(p), ctypes.byref(stride)))
        return p.value, stride.value

    def stream(self) -> int:
        return lib().vf_mpm3_stream(self._h)

    def set_schedule(self, schedule: int) -> None:
        check(lib().vf_mpm3_set_p2g(self._h, schedule))

    def fixed_grid(self) -> list:
        """The last scatter's exact grid (VF_P2G_FIXED): m, mu, mv, mw as int64 with 40 fractional bits."""
        n = self._nx * self._ny * self._nz
        out = []
        for f in range(4):
            a = np.empty(n, np.int64)
            check(lib().vf_mpm3_read_fixed(self._h, f, a.ctypes.data_as(_i64p), n))
            out.append(a)
        return out

    def snapshot(self) -> bytes:
        """The simulation's state as a versioned, checksummed blob (particles in their current order, params,
        the last grid, the step count)."""
        return _snapshot(lib().vf_mpm3_snapshot, self._h)

    def restore(self, blob: bytes) -> None:
        """Resume from snapshot(); the grid, particle count and physics flags must match (ValueError otherwise)."""
        check(lib().vf_mpm3_restore(self._h, blob, len(blob)))

    def pool_used(self) -> int:
        out = ctypes.c_int32()
        check(lib().vf_mpm3_pool_used(self._h, ctypes.byref(out)))
        return out.value

    def schedule(self) -> int:
        """The scatter schedule the steps run (VF_P2G_AUTO resolved for this size)."""
        return int(lib().vf_mpm3_schedule(self._h))

    def set_fused(self, on: bool) -> None:
        """The fused step (the gather and the next step's scatter in one kernel) where it applies; off, the default,
        runs the separate tiled scatter and gather."""
        check(lib().vf_mpm3_set_fused(self._h, 1 if on else 0))

    def fused(self) -> bool:
        return bool(lib().vf_mpm3_fused(self._h))

    def set_graph(self, on: bool) -> None:
        """advance() replays its steps two at a time from a captured CUDA graph (off by default)."""
        check(lib().vf_mpm3_set_graph(self._h, 1 if on else 0))

    def pool_capacity(self) -> int:
        return int(lib().vf_mpm3_pool_capacity(self._h))

    def touched_nodes(self) -> int:
        out = ctypes.c_int64()
        check(lib().vf_mpm3_touched_nodes(self._h, ctypes.byref(out)))
        return out.value

    def profile(self, enable: bool) -> None:
        check(lib().vf_mpm3_profile(self._h, 1 if enable else 0))

    def profile_read(self):
        return _profile_read(lib().vf_mpm3_profile_read, self._h)

    def launches(self) -> int:
        return int(lib().vf_mpm3_launches(self._h))

    def particle_diagnostics(self, speed, sound, dt):
        out = (ctypes.c_double * 7)()
        check(lib().vf_mpm3_particle_diagnostics(self._h, speed, sound, dt, out))
        return list(out)

    def steps(self) -> int:
        return int(lib().vf_mpm3_steps(self._h))

    def close(self) -> None:
        if self._h:
            lib().vf_mpm3_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------------------------- shallow water

@dataclass(frozen=True)
class Advance:
    """PatchSimulation.Advance (PatchSimulation.java:33-39)."""
    steps: int
    spent_ticks: int
    behind_ticks: int

    def mean_step(self) -> float:
        return 0.0 if self.steps == 0 else seconds(self.spent_ticks) / self.steps


class LearnedSimulation:
    """The learned coarse shallow-water solver as one native handle (vf_swe_learned_*): an nx x ny coarse patch,
    the network's correction every `interval` ticks (`net` None: the plain coarse solver), and with a `threshold`
    the tiles whose depth jump exceeds it stepped by the fine solver. The same calls, in the same order, as
    learned.LearnedShallowWater."""

    def __init__(self, nx: int, ny: int, net: "FluxNet | None", interval: int, *, tile: int = 64,
                 threshold: float | None = None, margin: int = 8, dx: float = 1.0):
        h = _vp()
        check(lib().vf_swe_learned_create(nx, ny, net._h if net is not None else None, int(interval), tile,
                                          0 if threshold is None else 1,
                                          0.0 if threshold is None else float(threshold), margin, dx,
                                          ctypes.byref(h)))
        self._h, self.nx, self.ny, self.net = h, nx, ny, net

    def load(self, h, hu, hv) -> None:
        n = self.nx * self.ny
        a = [_f32(np.ravel(q), n) for q in (h, hu, hv)]
        check(lib().vf_swe_learned_load(self._h, *[_fp(q) for q in a]))

    def advance(self, ticks_: int) -> None:
        check(lib().vf_swe_learned_advance(self._h, int(ticks_)))

    def read(self):
        out = [np.empty(self.nx * self.ny, np.float32) for _ in range(3)]
        check(lib().vf_swe_learned_read(self._h, *[_fp(q) for q in out]))
        return [q.reshape(self.ny, self.nx) for q in out]

    def counts(self) -> tuple:
        """(coarse steps, corrections applied, fallback tiles stepped)."""
        out = (ctypes.c_int64 * 3)()
        check(lib().vf_swe_learned_counts(self._h, out))
        return tuple(out)

    def close(self) -> None:
        if self._h:
            lib().vf_swe_learned_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class PatchSimulation:
    """PatchSimulation (PatchSimulation.java): one shallow-water patch on the GPU, advanced by slices of time."""

    def __init__(self, nx: int, ny: int, edges: Sequence[int] = (EDGE_WALL,) * 4):
        e = np.ascontiguousarray(edges, np.int32)
        if e.shape != (4,):
            raise IllegalArgumentException(VF_EINVAL, "every side of a patch needs an edge")
        h = _vp()
        check(lib().vf_swe_create(nx, ny, _ip(e), ctypes.byref(h)))
        self._h = h
        self._nx, self._ny = nx, ny

    def nx(self):
        return self._nx

    def ny(self):
        return self._ny

    def on_gpu(self) -> bool:
        return bool(lib().vf_swe_on_gpu(self._h))

    def load(self, h, hu, hv, params) -> None:
        n = self._nx * self._ny
        a = [_f32(q, n) for q in (h, hu, hv)]
        w = _words(params)
        check(lib().vf_swe_load(self._h, *[_fp(q) for q in a], _ip(w), len(w)))

    def params(self, params) -> None:
        w = _words(params)
        check(lib().vf_swe_params(self._h, _ip(w), len(w)))

    def device_state(self):
        """Device pointers (h, hu, hv) of the current state, valid until the next dispatch."""
        p = [_vp() for _ in range(3)]
        check(lib().vf_swe_state(self._h, *[ctypes.byref(q) for q in p]))
        return p

    def measure_speed(self) -> None:
        check(lib().vf_swe_measure_speed(self._h))

    def restrict_from(self, fine: "PatchSimulation") -> None:
        """This (coarse) state = the fine state averaged over 2x2 cells."""
        check(lib().vf_swe_restrict(fine._h, self._h))

    def prolong_from(self, coarse: "PatchSimulation", x0: int, y0: int) -> None:
        """This patch's cells copied from coarse cells from (x0, y0) on, each to its 2x2 fine cells."""
        check(lib().vf_swe_prolong(coarse._h, x0, y0, self._h))

    def restrict_into(self, fx0: int, fy0: int, coarse: "PatchSimulation", x0: int, y0: int, nx: int, ny: int) -> None:
        """nx x ny coarse cells from (x0, y0) = this patch's 2x2 means from its cell (fx0, fy0)."""
        check(lib().vf_swe_restrict_patch(self._h, fx0, fy0, coarse._h, x0, y0, nx, ny))

    def copy_from(self, other: "PatchSimulation") -> None:
        check(lib().vf_swe_copy_state(self._h, other._h))

    def jump_indicator(self, tile: int) -> np.ndarray:
        """Per tile (rows of tiles from the south-west): the largest relative depth jump between neighbours."""
        tx, ty = -(-self._nx // tile), -(-self._ny // tile)
        out = np.empty(tx * ty, np.float32)
        check(lib().vf_swe_jump_indicator(self._h, tile, _fp(out), len(out)))
        return out.reshape(ty, tx)

    def advance(self, ticks_: int, max_steps: int) -> Advance:
        steps = ctypes.c_int32()
        spent = ctypes.c_int64()
        behind = ctypes.c_int64()
        check(lib().vf_swe_advance(self._h, ticks_, max_steps, ctypes.byref(steps), ctypes.byref(spent),
                                   ctypes.byref(behind)))
        return Advance(steps.value, spent.value, behind.value)

    def read(self):
        n = self._nx * self._ny
        out = [np.empty(n, np.float32) for _ in range(3)]
        check(lib().vf_swe_read(self._h, *[_fp(o) for o in out]))
        return out

    def fastest_wave(self) -> float:
        v = ctypes.c_double()
        check(lib().vf_swe_fastest_wave(self._h, ctypes.byref(v)))
        return v.value

    def allowed_step(self, courant, dx, dy) -> float:
        f = self.fastest_wave()
        return courant * min(dx, dy) / f if f > 0 else 0.0

    def clamped(self) -> int:
        v = ctypes.c_int32()
        check(lib().vf_swe_clamped(self._h, ctypes.byref(v)))
        return v.value

    def now(self) -> int:
        return int(lib().vf_swe_now(self._h))

    def steps(self) -> int:
        return int(lib().vf_swe_steps(self._h))

    # the raw rotation, for the reference test harness (Stepper.java)
    def dispatch(self, n: int = 1) -> None:
        check(lib().vf_swe_dispatch(self._h, n))

    def dispatched(self) -> int:
        return int(lib().vf_swe_dispatched(self._h))

    def write_budget(self, slot: int, ticks_: int) -> None:
        check(lib().vf_swe_write_budget(self._h, slot, ticks_))

    def set_tile_width(self, width: int) -> None:
        """The exact mode's step kernel: 64 (the default) or 32 the staged tile kernel of that width, 0 the column
        walk over strips. Results do not depend on it."""
        check(lib().vf_swe_set_tile_width(self._h, width))

    def tile_width(self) -> int:
        return int(lib().vf_swe_tile_width(self._h))

    def set_overlap(self, on: bool) -> None:
        """Steps launched as programmatic dependents of the previous step (default) or in plain stream order."""
        check(lib().vf_swe_set_overlap(self._h, 1 if on else 0))

    def set_exact(self, on: bool) -> None:
        """The reference's strict f32 arithmetic, bit for bit (default), or the fast mode (fused multiply-adds and
        approximate reciprocals, within a stated tolerance)."""
        check(lib().vf_swe_set_exact(self._h, 1 if on else 0))

    def exact(self) -> bool:
        return bool(lib().vf_swe_exact(self._h))

    def snapshot(self) -> bytes:
        """The patch's state as a versioned, checksummed blob (cells, speed and budget words, clock, steps)."""
        return _snapshot(lib().vf_swe_snapshot, self._h)

    def restore(self, blob: bytes) -> None:
        """Resume from snapshot(); the patch's size and edges must match (ValueError otherwise)."""
        check(lib().vf_swe_restore(self._h, blob, len(blob)))

    def read_budget(self, slot: int) -> int:
        v = ctypes.c_int32()
        check(lib().vf_swe_read_budget(self._h, slot, ctypes.byref(v)))
        return v.value

    def diagnostics(self, g, dry, dt, dx, dy):
        """Diagnostics.of(h, hu, hv, g, dry, dt, dx, dy) of the current state, reduced on the device."""
        out = (ctypes.c_double * 9)()
        check(lib().vf_swe_diagnostics(self._h, g, dry, dt, dx, dy, out))
        return list(out)

    def profile(self, enable: bool) -> None:
        check(lib().vf_swe_profile(self._h, 1 if enable else 0))

    def profile_read(self):
        return _profile_read(lib().vf_swe_profile_read, self._h)

    def launches(self) -> int:
        return int(lib().vf_swe_launches(self._h))

    def stream(self) -> int:
        return lib().vf_swe_stream(self._h)

    def close(self) -> None:
        if self._h:
            lib().vf_swe_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
