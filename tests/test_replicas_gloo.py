"""Multi-rank plumbing of bench.py on CPU (gloo, world size 2): every rank
runs its own replica and the timed value is the max over ranks."""
import os
import socket
import subprocess
import sys
import textwrap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = textwrap.dedent("""
    import os, sys
    sys.path.insert(0, {root!r})
    import torch
    import bench
    world, rank, local = bench.dist_env()
    dist = bench.init_dist(world, "gloo")
    ms = 10.0 + 5.0 * rank                      # rank 1 is the slow one
    m = bench.max_over_ranks(dist, ms, torch.device("cpu"))
    assert m == 15.0, m
    dist.barrier()
    dist.destroy_process_group()
    print("rank", rank, "max", m)
""")


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_max_over_ranks_gloo(tmp_path):
    script = tmp_path / "worker.py"
    script.write_text(WORKER.format(root=ROOT))
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, WORLD_SIZE="2", RANK=str(rank), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        procs.append(subprocess.Popen([sys.executable, str(script)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT, text=True))
    outs = [p.communicate(timeout=120)[0] for p in procs]
    for p, o in zip(procs, outs):
        assert p.returncode == 0, o
    assert all("max 15.0" in o for o in outs)
