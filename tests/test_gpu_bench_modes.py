"""bench.py --io on a small block: one JSON line with every IO timing, the
record counts and file sizes it reports, and the CPU restatement's timing."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_io_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--io", "--workload", "block250k",
                        "--warmup", "3"], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])
    t = line["seconds"]
    for k in ("frame_full", "frame_partial", "save_frame_full", "save_frame_partial", "download",
              "download_pinned", "save_snapshot", "read_snapshot", "upload", "upload_pinned"):
        assert t[k] > 0, k
    n = line["config"]["particles"]
    assert line["records"]["full"] == n
    assert line["bytes"]["soa"] == 28 * 8 * n
    assert line["file_bytes"]["snapshot"] > line["bytes"]["soa"]
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["frame_full"] > 0
