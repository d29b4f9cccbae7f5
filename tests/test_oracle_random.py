"""The java.util.Random restatement against values the JDK is known to produce, and the
Python and C restatements against each other."""
import ctypes

import numpy as np

from _oracle import JavaRandom, lib, OrPhysics  # noqa: F401


def test_known_jdk_values():
    # new Random(42).nextInt() and nextGaussian() as the JDK returns them
    assert JavaRandom(42).next_int() == -1170105035
    assert JavaRandom(42).next_gaussian() == 1.1419053154730547
    # nextInt(bound) for a power of two and otherwise
    r = JavaRandom(42)
    assert [r.next_int(10) for _ in range(5)] == [0, 3, 8, 4, 0]


def test_python_and_c_agree():
    from _oracle import ORACLE_DIR  # noqa: F401

    class JR(ctypes.Structure):
        _fields_ = [("seed", ctypes.c_int64), ("have", ctypes.c_int), ("g", ctypes.c_double)]

    L = lib()
    L.or_jrand_init.argtypes = [ctypes.POINTER(JR), ctypes.c_int64]
    L.or_jrand_float.argtypes = [ctypes.POINTER(JR)]
    L.or_jrand_float.restype = ctypes.c_float
    L.or_jrand_gaussian.argtypes = [ctypes.POINTER(JR)]
    L.or_jrand_gaussian.restype = ctypes.c_double
    L.or_jrand_int.argtypes = [ctypes.POINTER(JR), ctypes.c_int32]
    L.or_jrand_int.restype = ctypes.c_int32
    for seed in (0, 3, 71, 123456789, -5):
        c = JR()
        L.or_jrand_init(ctypes.byref(c), seed)
        p = JavaRandom(seed)
        for k in range(200):
            if k % 3 == 0:
                assert np.float32(L.or_jrand_float(ctypes.byref(c))) == p.next_float()
            elif k % 3 == 1:
                assert L.or_jrand_gaussian(ctypes.byref(c)) == p.next_gaussian()
            else:
                assert L.or_jrand_int(ctypes.byref(c), 1000 + k) == p.next_int(1000 + k)
