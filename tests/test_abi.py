"""The C-ABI library loads and exports every entry point include/*.h declares (no GPU needed), and the
host-side argument checks the reference's constructors make are refused before any device work."""
import ctypes
import pathlib
import re
import subprocess

import pytest

import vexfluid

ROOT = pathlib.Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b(vf_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def exported_symbols(so):
    out = subprocess.run(["nm", "-D", "--defined-only", str(so)], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_library_exports_every_declared_entry_point():
    so = vexfluid.LIBRARY
    if not so.exists():
        vexfluid.build()
    decl = declared_symbols()
    assert len(decl) > 40
    missing = [d for d in decl if d not in exported_symbols(so)]
    assert not missing, f"declared but not exported: {missing}"
    L = vexfluid.lib()
    for d in decl:
        assert getattr(L, d) is not None


def test_binary_version_needs_a_device():
    """vf_binary_version reports the architecture the runtime sees for the library's kernels; without a device it
    is VF_ENODEV (the GPU test checks the value)."""
    L = vexfluid.lib()
    v = ctypes.c_int32(0)
    rc = L.vf_binary_version(ctypes.byref(v))
    if L.vf_device_ok():
        assert rc == 0 and v.value == 100, (rc, v.value)
    else:
        assert rc == vexfluid.VF_ENODEV


@pytest.mark.gpu
def test_library_runs_sm100a_code():
    """The runtime loads the library's kernels as sm_100 binaries (cudaFuncAttributes.binaryVersion 100)."""
    L = vexfluid.lib()
    v = ctypes.c_int32(0)
    assert L.vf_binary_version(ctypes.byref(v)) == 0, vexfluid.last_error()
    assert v.value == 100


def test_oversized_grids_are_refused_before_the_device():
    """Cell keys are int32 in the kernels: grids whose keys would overflow are refused with VF_EINVAL, whatever
    the device."""
    L = vexfluid.lib()
    h = ctypes.c_void_p()
    assert L.vf_mpm2_create(50000, 50000, 10, 0, ctypes.byref(h)) == vexfluid.VF_EINVAL
    assert "2^31" in vexfluid.last_error()
    assert L.vf_mpm3_prepare(2048, 2048, 1024, 10, 0, ctypes.byref(h)) == vexfluid.VF_EINVAL
    assert "int32" in vexfluid.last_error()
    f = (ctypes.c_float * 1)(0.5)
    i = (ctypes.c_int32 * 1)(0)
    one = ctypes.c_int64(1)
    assert L.vf_sort2(50000, 50000, f, f, one, i, i) == vexfluid.VF_EINVAL
    assert L.vf_sort2_noalloc(50000, 50000, f, f, one, i, i) == vexfluid.VF_EINVAL


def test_argument_checks_come_before_the_device():
    """Flip3Step/FlipStep refuse particles < 1, Scatter refuses grids under 2 nodes (FlipStep.java:86-88,
    Flip3Step.java:54-56, Scatter.java:516-520, ShallowWater.java:167-169), whatever the device."""
    L = vexfluid.lib()
    h = ctypes.c_void_p()
    assert L.vf_mpm2_create(32, 32, 0, 0, ctypes.byref(h)) == vexfluid.VF_EINVAL
    assert "needs particles" in vexfluid.last_error()
    assert L.vf_mpm3_prepare(24, 24, 24, 0, 0, ctypes.byref(h)) == vexfluid.VF_EINVAL
    edges = (ctypes.c_int32 * 4)(0, 0, 0, 0)
    assert L.vf_swe_create(0, 5, edges, ctypes.byref(h)) == vexfluid.VF_EINVAL
    bad = (ctypes.c_int32 * 4)(0, 0, 7, 0)
    assert L.vf_swe_create(5, 5, bad, ctypes.byref(h)) == vexfluid.VF_EINVAL
    with pytest.raises(vexfluid.IllegalArgumentException):
        vexfluid.flip_params(0, 0, -10, 1, 1)
    with pytest.raises(vexfluid.IllegalArgumentException):
        vexfluid.flip3_params(0.01, 0, -10, 0, -1, 1)
    with pytest.raises(vexfluid.IllegalArgumentException):
        vexfluid.swe_params(9.81, 0.51, 1, 1)
    vexfluid.swe_params(9.81, 0.9, 1, 1, allow_instability=True)


def test_no_device_is_an_error_not_a_fallback():
    """Without a CUDA device the library refuses work with VF_ENODEV: there is no CPU path."""
    L = vexfluid.lib()
    if L.vf_device_ok():
        pytest.skip("a CUDA device is present")
    h = ctypes.c_void_p()
    assert L.vf_mpm2_create(32, 32, 10, 0, ctypes.byref(h)) == vexfluid.VF_ENODEV
    with pytest.raises(vexfluid.VfError):
        vexfluid.ParticleSimulation(32, 32, 10)


def test_the_learned_handle_is_created_or_refused_cleanly():
    """vf_swe_learned_create through its declared signature: a handle where there is a device, VF_ENODEV where there
    is none; never a crash."""
    import ctypes
    import vexfluid as vf
    h = ctypes.c_void_p()
    rc = vf.lib().vf_swe_learned_create(64, 64, None, 1000, 16, 1, 0.5, 4, 1.0, ctypes.byref(h))
    if rc == 0:
        vf.lib().vf_swe_learned_destroy(h)
    else:
        assert rc == vf.VF_ENODEV, rc
        assert not h.value
