"""The N > 1 host path of bench.py on CPU ranks over gloo (world size 2):
rank 0 alone prints one JSON line, every rank exits 0, and the timing
reduction is the max over ranks."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_reference_arm_two_gloo_ranks():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="1")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", f"--master-port={_free_port()}", str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3", "--grid-n", "16"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"


def _max_worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sys.path.insert(0, str(ROOT))
    import bench

    got = bench.max_over_ranks(dist, float(10 * (rank + 1)), 0)
    bench.barrier(dist, 0)
    q.put((rank, got))
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_max_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 20.0), (1, 20.0)]


def test_bench_error_helpers():
    """bench.py's precision comparison: per-field RMS / max relative errors
    and the velocity error by bands of levels, on known arrays."""
    import numpy as np

    sys.path.insert(0, str(ROOT))
    import bench

    rng = np.random.default_rng(0)
    b = {n: rng.normal(size=(16, 4, 4)) for n in bench.COMPARED}
    a = {n: b[n].copy() for n in bench.COMPARED}
    a["u"][12:] += 0.5  # levels 13..16 of 16: the top band of four
    err = bench.field_errors(a, b)
    assert err["v"] == {"rms_rel": 0.0, "max_rel": 0.0}
    rms_b = np.sqrt((b["u"] ** 2).mean())
    assert abs(err["u"]["rms_rel"] - np.sqrt(0.25 * 0.25) / rms_b) < 1e-12
    bands = bench.level_band_errors(a, b, nbands=4)
    assert bands["v"] == [0.0] * 4 and bands["w"] == [0.0] * 4
    assert bands["u"][:3] == [0.0] * 3
    assert abs(bands["u"][3] - round(0.5 / rms_b, 5)) < 1e-12
