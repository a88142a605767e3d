"""bench.py pieces that run without a GPU: the replica aggregation over
world_size-2 gloo ranks, and the reference arm's JSON line."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from howtest import REPO, REF_BIN

sys.path.insert(0, str(REPO))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    per_rank_ms = [100.0, 250.0][rank]
    ms = bench.max_over_ranks(per_rank_ms, world, "cpu")
    q.put((rank, ms, bench.replica_value(world, 64 ** 3, 10, ms)))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank, ms, value in res:
        assert ms == 250.0   # the slowest replica sets the time
        assert value == pytest.approx(2 * 64 ** 3 * 10 / 0.25)


@pytest.mark.skipif(not REF_BIN.exists(), reason="reference build absent")
def test_reference_arm_prints_contract_line():
    """The reference arm runs the reference's own build on the headline
    problem without this library: pointed at a library path that does not
    exist, it must still succeed.  Its `config` is our arm's."""
    env = dict(os.environ, HOW_MHD_LIB="/nonexistent/libhowmhd.so")
    r = subprocess.run([sys.executable, str(REPO / "bench.py"), "--impl", "reference", "--steps", "2",
                        "--warmup", "0", "--ref-sizes", ""], capture_output=True, text=True, timeout=600, cwd=REPO,
                       env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "zone-cycles/s"
    assert line["cpu_baseline"]["kind"] == "reference" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["value"] > 0
    assert line["steps"] == 2 and line["sample"]["steps"] == 2
    import bench
    assert line["config"] == bench.headline_config(256, 1)
