"""bench.py's multi-process plumbing on CPU (gloo, world size 2): the max/sum reductions the
timing uses, and the reference arm launched under torchrun, where rank 0 alone measures and
prints one JSON line and the other rank exits 0 without output."""
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, port, out_dir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": "2",
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    import bench

    d = bench.Dist(want_gpu=False)
    try:
        d.barrier()
        res = {"backend": d.backend, "max": d.reduce(10.0 + rank, "max"), "sum": d.reduce(1.0 + rank, "sum"),
               "world": d.world, "rank": d.rank}
        d.barrier()
    finally:
        d.close()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump(res, f)


def test_dist_reductions_two_ranks(tmp_path):
    mp.spawn(_rank, args=(_free_port(), str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        res = json.load(open(tmp_path / f"rank{r}.json"))
        assert res == {"backend": "gloo", "max": 11.0, "sum": 3.0, "world": 2, "rank": r}


def test_reference_arm_under_torchrun(built):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference",
           "--particles", "3000", "--steps", "1", "--warmup", "1"]
    p = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [x for x in p.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, p.stdout[-2000:]
    out = json.loads(lines[0])
    assert out["impl"] == "reference" and out["value"] > 0 and out["e2e"]["h2d_bytes_per_step"] == 0
    assert out["cpu_baseline"]["kind"] == "reference"
    assert out["product_library_loaded"] is False  # inputs come from the oracle's generator
    assert out["config"]["seeds"] == [7, 8, 9, 10]  # the GPU arm's particle sets
