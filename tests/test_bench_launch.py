"""bench.py --gpus N launches N ranks itself when it is started outside a
launcher: each rank joins one process group (gloo here, on the CPU) and the
group has N members.  `python bench.py --gpus N` on a multi-GPU node relies on
this path."""
import json
import os
import re
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_bench_launches_its_ranks():
    env = dict(os.environ)
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2", "--probe-ranks"], cwd=ROOT,
                         env=env, capture_output=True, text=True, timeout=240)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(m) for m in re.findall(r"\{[^{}]*\}", out.stdout)]
    assert sorted(ln["rank"] for ln in lines) == [0, 1], out.stdout
    for ln in lines:
        assert ln["world_size"] == 2 and ln["ranks_seen"] == 2 and ln["group_size"] == 2, ln
