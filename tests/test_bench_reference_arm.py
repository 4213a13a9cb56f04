"""bench.py's reference arm as torchrun starts it: rank 0 alone times the reference's CPU sweep, on every
core the process may run on although torchrun sets OMP_NUM_THREADS=1 for each rank, and prints the same
config and scaling as the GPU arm at that N; the other ranks exit 0 and print nothing.  CPU only."""
import json
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(REPO, "oracle", "_ref", "libidcref.so")


def _run(rank: int, world: int, *extra: str) -> subprocess.CompletedProcess:
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), OMP_NUM_THREADS="1")
    cmd = [sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--gpus", str(world),
           "--steps", "1", "--warmup", "1", "--nx", "32", *extra]
    return subprocess.run(cmd, env=env, cwd=REPO, capture_output=True, text=True, timeout=300)


def test_reference_arm_other_ranks_exit_without_work():
    r = _run(1, 2)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference library not built")
@pytest.mark.parametrize("mode,parallelism,scaling", [("partitioned", "ordinates2", "strong"),
                                                      ("replicas", "replicas2", "weak")])
def test_reference_arm_rank0_uses_every_core_and_mirrors_the_config(mode, parallelism, scaling):
    r = _run(0, 2, "--mode", mode)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["cpu_baseline"]["cores"] == len(os.sched_getaffinity(0))
    assert line["config"]["parallelism"] == parallelism
    assert line["scaling"] == scaling
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["value"] > 0
