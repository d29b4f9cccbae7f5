"""The 3D step with sparse grid storage (a page table of 8^3-node bricks over a pool) on the GPU.

Parity bars (tolerances written here), the dense tiled schedule's own:
* the grid after one scatter: per node |gpu - oracle| <= 1e-5 * max(1, |oracle|);
* positions after 100 steps: |gpu - oracle| <= 1e-4 * |oracle| per coordinate, particles matched by mass tags;
* the bricks a step takes from the pool: exactly the node bricks its particles' stencils reach.
"""
import numpy as np
import pytest

import vexfluid as vf
from _oracle import F, Flip3State, flip3_params, key3
from test_gpu_mpm3 import dam3
from test_gpu_tension3 import ball

pytestmark = pytest.mark.gpu

GRID = ("gm", "gmu", "gmv", "gmw")


def reached_bricks(x, y, z, nx, ny, nz):
    """The node bricks (8^3 nodes) the particles' stencils reach: each stencil cell's 8^3-cell brick, whose nodes
    run 10 along each axis, reaches its own node brick and the next one each way, within the domain."""
    nbx, nby = (nx - 2 + 7) // 8, (ny - 2 + 7) // 8
    pnx, pny, pnz = (nx + 7) // 8, (ny + 7) // 8, (nz + 7) // 8
    bricks = np.unique(key3(x, y, z, nx, ny, nz) >> 9)
    reached = set()
    for b in bricks:
        bx, by, bz = b % nbx, (b // nbx) % nby, b // (nbx * nby)
        for o in range(8):
            px, py, pz = bx + (o & 1), by + ((o >> 1) & 1), bz + (o >> 2)
            if px < pnx and py < pny and pz < pnz:
                reached.add((pz * pny + py) * pnx + px)
    return len(reached)


def check_grid(grid, o, tag):
    for f, key in enumerate(GRID):
        e = o.g[key].astype(np.float64)
        err = np.abs(grid[f] - e)
        assert np.all(err <= 1e-5 * np.maximum(1, np.abs(e))), (tag, key, float(err.max()))


def check_positions(pos, mass, o, tag):
    dev = np.argsort(mass.view(np.int32))
    ora = np.argsort(o.a["m"].view(np.int32))
    assert np.array_equal(mass.view(np.int32)[dev], o.a["m"].view(np.int32)[ora])
    for a, key in enumerate(("x", "y", "z")):
        e = o.a[key][ora]
        err = np.abs(pos[a][dev] - e)
        assert np.all(err <= 1e-4 * np.abs(e)), (tag, key, float((err / np.abs(e)).max()))


def test_a_sparse_step_matches_the_oracle():
    """Flip3Test's slab (seed 71): the grid after one step per node, the bricks it took, and 100 steps' positions."""
    n = 24
    x, y, z, m, p, _ = dam3(n, tagged=True)
    o = Flip3State(n, n, n, x, y, z, m)
    with vf.ParticleSimulation3(n, n, n, len(x), pool_bricks=27) as s:
        assert s.pool_capacity() == 27
        s.load([x, y, z], [np.zeros_like(x)] * 3, m, vf.flip3_params(*p))
        s.advance(1)
        assert s.pool_used() == reached_bricks(x, y, z, n, n, n)
        o.step(flip3_params(*p))
        check_grid(s.grid(), o, "one step")
        s.advance(99)
        for _ in range(99):
            o.step(flip3_params(*p))
        check_positions(s.positions(), s.read("m"), o, "100 steps")
        assert np.array_equal(np.sort(s.read("m").view(np.int32)), np.sort(m.view(np.int32)))


def test_a_blob_in_a_wide_domain_costs_only_the_bricks_it_reaches():
    """A ball of water falling through a 120^3 domain (3,375 brick positions) in a pool of 40 bricks: the grid's
    memory is 40 x 8 KB a pool against 27.6 MB for the dense box, and the run follows the oracle's dense box."""
    n = 120
    x, y, z, m = ball(n, n, n, (60.0, 90.0, 60.0), 5.0, seed=3)
    m = (m.view(np.int32) + np.arange(len(m), dtype=np.int32)).view(F)
    p = (2e-3, 0.0, -200.0, 0.0, 400.0, 1.0)
    o = Flip3State(n, n, n, x, y, z, m)
    with vf.ParticleSimulation3(n, n, n, len(x), pool_bricks=40) as s:
        s.load([x, y, z], [np.zeros_like(x)] * 3, m, vf.flip3_params(*p))
        used = []
        for _ in range(30):
            s.advance(1)
            used.append(s.pool_used())
        pos, mass = s.positions(), s.read("m")
    for _ in range(30):
        o.step(flip3_params(*p))
    check_positions(pos, mass, o, "30 steps")
    assert max(used) <= 40 and min(used) >= 8
    assert float(pos[1].mean()) < float(y.mean()) - 0.2   # it fell


def test_the_readouts_see_the_sparse_grid_as_a_box():
    """Flip3Test's conservation particles scattered once (sort, clear, scatter): every grid readout of the sparse
    handle is the dense handle's within the per-node bar, and both hold the particles' mass."""
    from test_gpu_mpm3 import conservation_inputs
    n = 14
    x, y, z, m, j, vel, c = conservation_inputs(n)
    fields = {"u": vel[0], "v": vel[1], "w": vel[2], "j": j}
    fields.update({f"c{a // 3}{a % 3}": c[a] for a in range(9)})
    out = []
    for kw in ({}, {"pool_bricks": 8}):
        with vf.ParticleSimulation3(n, n, n, len(x), **kw) as s:
            s.load([x, y, z], [vel[0], vel[1], vel[2]], m, vf.flip3_params(0.01, 0, -10, 0, 1e4, 1))
            for k, v in fields.items():
                s.write(k, v)
            s.run(vf.VF3_PASS_SORT | vf.VF3_PASS_CLEAR | vf.VF3_PASS_SCATTER)
            out.append([s.read(k) for k in GRID + ("gu", "gv", "gw")] + [s.touched_nodes()])
    for f in range(7):
        e = out[0][f].astype(np.float64)
        assert np.all(np.abs(out[1][f] - e) <= 1e-5 * np.maximum(1, np.abs(e))), f
    assert out[0][7] == out[1][7]
    assert abs(float(out[1][0].astype(np.float64).sum()) - float(m.astype(np.float64).sum())) <= 1e-4 * m.sum()


def test_a_pool_too_small_is_reported_not_overrun():
    n = 24
    x, y, z, m, p, _ = dam3(n)
    need = reached_bricks(x, y, z, n, n, n)
    with vf.ParticleSimulation3(n, n, n, len(x), pool_bricks=need - 2) as s:
        s.load([x, y, z], [np.zeros_like(x)] * 3, m, vf.flip3_params(*p))
        s.advance(1)
        with pytest.raises(vf.VfError, match="pool"):
            s.finish()
    with vf.ParticleSimulation3(n, n, n, len(x), pool_bricks=need) as s:
        s.load([x, y, z], [np.zeros_like(x)] * 3, m, vf.flip3_params(*p))
        s.advance(1)
        s.finish()
        assert s.pool_used() == need


def test_sparse_storage_refuses_what_it_does_not_run():
    with pytest.raises(ValueError):
        vf.ParticleSimulation3(16, 16, 16, 10, pool_bricks=8, schedule=vf.VF_P2G_ATOMIC)
    with pytest.raises(ValueError):
        vf.ParticleSimulation3(16, 16, 16, 10, pool_bricks=8, tension=True)
    with pytest.raises(ValueError):
        vf.ParticleSimulation3(16, 16, 16, 10, pool_bricks=0)
    with vf.ParticleSimulation3(16, 16, 16, 10, pool_bricks=1000) as s:
        assert s.pool_capacity() == 8       # cut to the domain's 2 x 2 x 2 bricks
        with pytest.raises(ValueError):
            s.set_schedule(vf.VF_P2G_FIXED)
    with vf.ParticleSimulation3(16, 16, 16, 10) as d:
        with pytest.raises(vf.IllegalStateException):
            d.pool_used()


def test_a_dense_snapshot_resumes_in_sparse_storage():
    n = 24
    x, y, z, m, p, _ = dam3(n, tagged=True)
    with vf.ParticleSimulation3(n, n, n, len(x)) as a:
        a.load([x, y, z], [np.zeros_like(x)] * 3, m, vf.flip3_params(*p))
        a.advance(5)
        blob = a.snapshot()
        grid = a.grid()
    with vf.ParticleSimulation3(n, n, n, len(x), pool_bricks=27) as b:
        b.restore(blob)
        for f, g in enumerate(b.grid()):
            assert np.array_equal(g.view(np.int32), grid[f].view(np.int32)), f
        b.advance(5)
        assert b.steps() == 10
        assert np.array_equal(np.sort(b.read("m").view(np.int32)), np.sort(m.view(np.int32)))
        again = b.snapshot()
    with vf.ParticleSimulation3(n, n, n, len(x)) as c:
        c.restore(again)
        assert c.steps() == 10


def test_several_blobs_share_one_pool():
    """Four separated balls in one 160^3 domain are more bricks of the same pool, stepped by the same launches: the
    pool holds each blob's bricks (the sum, as they are far apart), and 20 steps follow the oracle's dense box."""
    n = 160
    centres = [(30.0, 40.0, 30.0), (120.0, 40.0, 40.0), (40.0, 100.0, 120.0), (120.0, 120.0, 110.0)]
    parts = [ball(n, n, n, c, 6.0, seed=k) for k, c in enumerate(centres)]
    x, y, z, m = (np.concatenate([p[a] for p in parts]) for a in range(4))
    m = (m.view(np.int32) + np.arange(len(m), dtype=np.int32)).view(F)
    each = sum(reached_bricks(p[0], p[1], p[2], n, n, n) for p in parts)
    assert reached_bricks(x, y, z, n, n, n) == each
    p = (2e-3, 0.0, -100.0, 0.0, 400.0, 1.0)
    o = Flip3State(n, n, n, x, y, z, m)
    with vf.ParticleSimulation3(n, n, n, len(x), pool_bricks=each + 16) as s:
        s.load([x, y, z], [np.zeros_like(x)] * 3, m, vf.flip3_params(*p))
        s.advance(1)
        assert s.pool_used() == each
        s.advance(19)
        pos, mass = s.positions(), s.read("m")
    for _ in range(20):
        o.step(flip3_params(*p))
    check_positions(pos, mass, o, "four blobs, 20 steps")
