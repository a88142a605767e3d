"""The z-slab decomposition plan (how_part_plan, host only) on world_size 2
and 3 gloo ranks: every rank holds its slab of a padded field in the device
layout (x fastest, so a z plane is contiguous), fills its x/y ghosts and its
physical z sides, and exchanges the halo planes the plan names with its
neighbours over torch.distributed.  The result must equal the whole-domain
ghost fill (src/bound.cpp:19-107, x then y then z) bit for bit, for periodic
and open z boundaries; the whole-domain fill restated here is itself pinned
to the oracle's bound."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from howtest import CPUOracle


def fill_axis(a, axis, periodic, sides=3):
    """Ghost fill of one axis of a padded array (3 ghosts per side), in place."""
    n = a.shape[axis] - 6
    sl = lambda k: tuple(slice(None) if d != axis else k for d in range(a.ndim))   # noqa: E731
    if sides == 3 and periodic:
        src = [a[sl(s)].copy() for s in (n, n + 1, n + 2, 3, 4, 5)]
        for dst, v in zip((0, 1, 2, n + 3, n + 4, n + 5), src):
            a[sl(dst)] = v
        return
    if sides & 1:
        for d in (0, 1, 2):
            a[sl(d)] = a[sl(3)]
    if sides & 2:
        for d in (n + 3, n + 4, n + 5):
            a[sl(d)] = a[sl(n + 2)]


def fill_whole(a, bc):
    """x, then y, then z (device layout [k][j][i]: x is the last axis)."""
    fill_axis(a, 2, bc[0] == "periodic")
    fill_axis(a, 1, bc[1] == "periodic")
    fill_axis(a, 0, bc[2] == "periodic")


def test_whole_domain_fill_matches_oracle():
    n = (7, 5, 9)
    bc = ("periodic", "open", "open")
    rng = np.random.default_rng(3)
    q = rng.standard_normal((8, n[0] + 6, n[1] + 6, n[2] + 6))   # reference layout (v, i, j, k)
    o = CPUOracle(*n, bc=bc)
    o.set_state(q, faceb=[np.zeros(q.shape[1:])] * 3)
    ref = o.get_q(0)
    for v in range(8):
        a = np.ascontiguousarray(q[v].transpose(2, 1, 0))   # -> [k][j][i]
        fill_whole(a, bc)
        np.testing.assert_array_equal(a.transpose(2, 1, 0), ref[v])


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, n, bc, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import how_mhd as hm
        periodic = bc[2] == "periodic"
        info = hm.part_plan(n[2], world, periodic, rank)
        rng = np.random.default_rng(11)
        glob = rng.standard_normal((n[2] + 6, n[1] + 6, n[0] + 6))
        want = glob.copy()
        fill_whole(want, bc)
        loc = glob[info.kstart: info.kstart + info.nz + 6].copy()   # stale ghosts included
        fill_axis(loc, 2, bc[0] == "periodic")
        fill_axis(loc, 1, bc[1] == "periodic")
        if info.z_sides:
            fill_axis(loc, 0, periodic, info.z_sides)
        k = info.nplanes
        reqs = []
        recv_lo = torch.empty(k, *loc.shape[1:], dtype=torch.float64)
        recv_hi = torch.empty(k, *loc.shape[1:], dtype=torch.float64)
        if info.hi_part >= 0:
            reqs.append(dist.isend(torch.from_numpy(loc[info.send_up_first: info.send_up_first + k].copy()),
                                   info.hi_part, tag=1))
            reqs.append(dist.irecv(recv_hi, info.hi_part, tag=2))
        if info.lo_part >= 0:
            reqs.append(dist.isend(torch.from_numpy(loc[info.send_down_first: info.send_down_first + k].copy()),
                                   info.lo_part, tag=2))
            reqs.append(dist.irecv(recv_lo, info.lo_part, tag=1))
        for r in reqs:
            r.wait()
        if info.lo_part >= 0:
            loc[info.recv_lo_first: info.recv_lo_first + k] = recv_lo.numpy()
        if info.hi_part >= 0:
            loc[info.recv_hi_first: info.recv_hi_first + k] = recv_hi.numpy()
        same = np.array_equal(loc, want[info.kstart: info.kstart + info.nz + 6])
        out.put((rank, bool(same), info.kstart, info.nz, info.z_sides))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("bc", [("periodic", "open", "periodic"), ("open", "periodic", "open")],
                         ids=["periodic_z", "open_z"])
def test_halo_exchange_equals_whole_domain_fill_gloo(world, bc):
    n = (6, 5, 13)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, n, bc, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert all(r[1] for r in res), res
    assert sum(r[3] for r in res) == n[2] and res[0][2] == 0
    if bc[2] == "open":   # only the outer parts fill a z side themselves
        assert [r[4] for r in res] == [1] + [0] * (world - 2) + [2]
    else:
        assert all(r[4] == 0 for r in res)
