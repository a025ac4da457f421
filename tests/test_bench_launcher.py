"""bench.py --gpus N without torchrun starts N rank processes itself (one per GPU, rendezvous on
127.0.0.1) and reports n_gpus from the process group actually formed, in both arms; checked on
the CPU with --dry-run (gloo: the group, a barrier and a max over ranks, no GPU work)."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _run(*args):
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_PORT")}
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), *args], capture_output=True, text=True,
                       timeout=300, env=env)
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    return r.returncode, lines, r.stderr


@pytest.mark.parametrize("impl", ["ours", "reference"])
@pytest.mark.parametrize("n", [1, 2])
def test_gpus_n_forms_n_ranks(impl, n):
    rc, lines, err = _run("--gpus", str(n), "--dry-run", "--impl", impl)
    assert rc == 0, err[-800:]
    assert len(lines) == 1, lines  # rank 0 alone prints
    d = json.loads(lines[0])
    assert d["n_gpus"] == n and d["max_rank"] == n - 1 and d["impl"] == impl
