"""advance() replayed from a captured CUDA graph (vf_mpm3_set_graph) on the GPU.

Parity bars (written here): under the exact scatter schedule, where a step is deterministic, the replayed run is
bit-exact against the same run launched kernel by kernel, including across a params change and a reload; under the
tiled schedule, with tension, and with sparse storage, positions after 40 steps are within 1e-4 relative of the
oracle, the dense schedule's bar.
"""
import numpy as np
import pytest

import vexfluid as vf
from _oracle import F, Flip3State, drop3, flip3_params, stable_step
from test_gpu_mpm3 import dam3

pytestmark = pytest.mark.gpu

FIELDS3 = ["x", "y", "z", "u", "v", "w", "m", "j"] + [f"c{a}{b}" for a in range(3) for b in range(3)]


def fields(s):
    return [s.read(f).view(np.int32).copy() for f in FIELDS3]


def test_replayed_steps_are_the_launched_steps_to_the_bit():
    n = 24
    x, y, z, m, p, _ = dam3(n, tagged=True)
    p2 = (p[0], 30.0, p[2] / 2, -20.0, p[4], p[5])
    x2, y2, z2, m2, _, _ = dam3(n, seed=5, tagged=True)
    runs = []
    for graph in (True, False):
        with vf.ParticleSimulation3(n, n, n, len(x), schedule=vf.VF_P2G_FIXED) as s:
            s.set_graph(graph)
            s.load([x, y, z], [np.zeros_like(x)] * 3, m, vf.flip3_params(*p))
            s.advance(7)
            s.advance(13)
            a = fields(s)
            s.params(vf.flip3_params(*p2))
            s.advance(10)
            b = fields(s)
            s.load([x2, y2, z2], [np.zeros_like(x2)] * 3, m2, vf.flip3_params(*p))
            s.advance(9)
            c = fields(s) + [g.view(np.int32).copy() for g in s.grid()]
            runs.append((a, b, c, s.steps(), s.launches()))
    for stage in range(3):
        for f, (u, v) in enumerate(zip(runs[0][stage], runs[1][stage])):
            assert np.array_equal(u, v), (stage, f)
    assert runs[0][3] == runs[1][3] == 9
    assert runs[0][4] == runs[1][4]


@pytest.mark.parametrize("kind", ["tile", "tension", "sparse"])
def test_replayed_steps_follow_the_oracle(kind):
    n = 40
    x, y, z, m, _ = drop3(n, radius=8.0)
    m = (m.view(np.int32) + np.arange(len(m), dtype=np.int32)).view(F)
    bulk = 200.0 ** 2
    p = (stable_step(bulk, 1, 20, 0.3), 0.0, -300.0, 0.0, bulk, 1.0, 0.01 * bulk * 8 if kind == "tension" else 0.0)
    kw = {"tension": True} if kind == "tension" else {"pool_bricks": 125} if kind == "sparse" else {}
    o = Flip3State(n, n, n, x, y, z, m)
    with vf.ParticleSimulation3(n, n, n, len(x), **kw) as s:
        s.set_graph(True)
        s.load([x, y, z], [np.zeros_like(x)] * 3, m, vf.flip3_params(*p))
        s.advance(40)
        pos, mass = s.positions(), s.read("m")
        assert s.steps() == 40
    for _ in range(40):
        o.step(flip3_params(*p), tension=kind == "tension")
    dev = np.argsort(mass.view(np.int32))
    ora = np.argsort(o.a["m"].view(np.int32))
    assert np.array_equal(mass.view(np.int32)[dev], o.a["m"].view(np.int32)[ora])
    for a, key in enumerate(("x", "y", "z")):
        e = o.a[key][ora]
        err = np.abs(pos[a][dev] - e)
        assert np.all(err <= 1e-4 * np.abs(e)), (kind, key, float((err / np.abs(e)).max()))
