"""k-point sharding host logic with world_size-2 gloo ranks on CPU."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from hack_wein2k_b200 import kshard


def test_assignment_covers_every_kpoint_once_and_balances():
    rng = np.random.default_rng(0)
    sizes = list(rng.integers(4400, 4750, size=64))
    for world in (1, 2, 3, 4, 8):
        parts = kshard.assign_kpoints(sizes, world)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(64))
        loads = [sum(sizes[k] ** 2 for k in p) for p in parts]
        assert max(loads) - min(loads) <= max(s ** 2 for s in sizes)


def test_batch_state_restarts_at_first_unfinished(tmp_path):
    path = str(tmp_path / "state.json")
    st = kshard.BatchState.load(path)
    st.mark(0, {"n": 10})
    st.mark(2, {"n": 12})
    st2 = kshard.BatchState.load(path)
    assert st2.todo([0, 1, 2, 3]) == [1, 3]
    calls = []
    out = kshard.run_sharded([10, 11, 12, 13], lambda k: calls.append(k) or {"n": 10 + k}, state=st2)
    assert calls == [1, 3] and sorted(out) == [0, 1, 2, 3]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, fail_k, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from hack_wein2k_b200 import lattice
    br2, ortho, pia = lattice.latgen("P", 6.0, 6.5, 7.0)
    ks = [np.array([0.1 * i, 0.05 * i, 0.0]) for i in range(6)]
    sizes = [len(lattice.coors(4.0, k, br2, ortho, pia)[4]) for k in ks]

    def worker(k):
        if k == fail_k:
            raise ValueError("planted failure")
        return {"nv": len(lattice.coors(4.0, ks[k], br2, ortho, pia)[4]), "rank": rank}

    try:
        out = kshard.run_sharded(sizes, worker, rank, world)
        q.put((rank, "ok", {k: v["nv"] for k, v in out.items()}, sizes))
    except kshard.KShardError as e:
        q.put((rank, "err", str(e), sizes))
    dist.destroy_process_group()


def _spawn(fail_k):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, fail_k, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    return sorted(res)


def test_two_gloo_ranks_gather_all_kpoints():
    res = _spawn(fail_k=-1)
    (r0, s0, out0, sizes), (r1, s1, out1, _) = res
    assert s0 == s1 == "ok"
    assert out0 == out1 == {k: sizes[k] for k in range(6)}


def test_failed_kpoint_is_reported_on_every_rank():
    res = _spawn(fail_k=3)
    assert all(r[1] == "err" and "k-point 3" in r[2] for r in res)


def _force_rank(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sizes = [40, 55, 47, 61, 52]
    weights = [0.1, 0.3, 0.2, 0.25, 0.15]
    local = torch.zeros(4, 3, dtype=torch.float64)
    for k in kshard.assign_kpoints(sizes, world)[rank]:
        g = torch.arange(12, dtype=torch.float64).reshape(4, 3) * (k + 1) - k  # stands in for dE_k/dPOS
        local += weights[k] * g
    q.put((rank, kshard.allreduce_forces(local).tolist()))
    dist.destroy_process_group()


def test_force_sum_over_ranks_equals_serial_sum():
    """Every rank gets the k-weighted force sum over all k-points (one
    all-reduce), equal to the serial sum."""
    import torch
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_force_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    weights = [0.1, 0.3, 0.2, 0.25, 0.15]
    ref = sum(w * (torch.arange(12, dtype=torch.float64).reshape(4, 3) * (k + 1) - k) for k, w in enumerate(weights))
    for _, out in res:
        assert np.allclose(np.array(out), ref.numpy(), rtol=0, atol=1e-12)
