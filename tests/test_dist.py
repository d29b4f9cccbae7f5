"""The N>1 host path of bench.py on CPU: two gloo ranks (world size 2, 127.0.0.1) take the bench's Dist plumbing
through its barrier, max-over-ranks and sum, and deal the batched scenes round-robin so that every scene is
stepped by exactly one rank. No GPU."""
import json
import os
import socket
import subprocess
import sys
import textwrap

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = textwrap.dedent("""
    import json, os, sys
    sys.path.insert(0, {root!r})
    import bench
    d = bench.Dist()
    d.barrier()
    rank, world = d.rank, d.world
    mx = d.max(float(rank + 1) * 10.0)
    sm = d.sum(float(rank + 1))
    scenes = list(range(bench.N_BATCH))
    mine = scenes[rank::world]
    total = d.sum(float(len(mine)))
    d.close()
    print(json.dumps({{"rank": rank, "world": world, "max": mx, "sum": sm, "total": total, "mine": mine[:3]}}))
""")


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_share_the_bench_plumbing(tmp_path):
    pytest.importorskip("torch.distributed")
    script = tmp_path / "child.py"
    script.write_text(CHILD.format(root=ROOT))
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        try:
            out, err = p.communicate(timeout=120)
        except subprocess.TimeoutExpired:
            p.kill()
            raise
        assert p.returncode == 0, err[-2000:]
        outs.append(json.loads(out.strip().splitlines()[-1]))
    outs.sort(key=lambda o: o["rank"])
    for o in outs:
        assert o["world"] == 2
        assert o["max"] == 20.0          # the max over ranks, as the bench times a step
        assert o["sum"] == 3.0           # the work summed over ranks
        assert o["total"] == 256.0       # every scene dealt to exactly one rank
    assert outs[0]["mine"] == [0, 2, 4] and outs[1]["mine"] == [1, 3, 5]
