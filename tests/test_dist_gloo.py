"""The multi-rank host logic of bench.py on CPU (world size 2, gloo): the
device time of a step is the maximum over ranks, the whole-job rate counts
every rank's work against that time (replicas, weak scaling), and the
reference arm runs and prints on rank 0 only while the other ranks exit 0."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, port: int, out_dir: str) -> None:
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": "2",
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, str(ROOT))
    import torch

    import bench

    world, r, local, pg = bench.dist_setup(2)
    try:
        cpu = torch.device("cpu")
        bench.barrier(pg, cpu)
        step_ms = bench.max_over_ranks(pg, 10.0 * (rank + 1), cpu)  # rank 1 is the slower one
        rate = bench.job_rate(32, world, step_ms)
        bench.barrier(pg, cpu)
        Path(out_dir, f"rank{rank}.json").write_text(json.dumps({"world": world, "rank": r, "ms": step_ms,
                                                                  "rate": rate}))
    finally:
        pg.destroy_process_group()


def test_max_over_ranks_and_job_rate_under_gloo(tmp_path):
    mp.start_processes(_rank_main, args=(_free_port(), str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    got = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(2)]
    for r, g in enumerate(got):
        assert g["world"] == 2 and g["rank"] == r
        assert g["ms"] == 20.0                    # the slowest rank's time on every rank
        assert g["rate"] == 32 * 2 / 0.020        # both ranks' queries over that time


def test_reference_arm_prints_once_under_torchrun():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0", "--cpu-sample-rows", "20000", "--rows", "1000000"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300,
                       env={**os.environ, "OMP_NUM_THREADS": "2"})
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [json.loads(l) for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, p.stdout
    assert lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2 and lines[0]["value"] > 0
