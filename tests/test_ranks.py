"""The multi-rank path of bench.py on the host: two gloo ranks share the
barrier and the max-over-ranks time of the replicas, and the reference arm
under torchrun prints one JSON line from rank 0 while the other rank exits
without work."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      LOCAL_RANK=str(rank))
    import bench
    r = bench.Ranks("gloo", device="cpu", timeout_s=60)
    r.barrier()
    m = r.max_over_ranks(1.5 * (rank + 1))
    r.barrier()
    r.close()
    with open(os.path.join(out_dir, "rank%d.txt" % rank), "w") as f:
        f.write(repr(m))


def test_max_over_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp
    port = free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for r in range(2):
        assert float(open(tmp_path / ("rank%d.txt" % r)).read()) == 3.0


def test_single_rank_is_local(monkeypatch):
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    monkeypatch.delenv("RANK", raising=False)
    import bench
    r = bench.Ranks("gloo", device="cpu")
    assert r.world == 1 and r.dist is None
    assert r.max_over_ranks(2.5) == 2.5
    r.barrier()
    r.close()


@pytest.mark.timeout(600)
def test_reference_arm_under_torchrun():
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "1", "--cells", "32"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["n_gpus"] == 2
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
