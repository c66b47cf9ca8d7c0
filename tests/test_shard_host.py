"""Multi-GPU host logic of batched instances (realmolecule_b200.shard), run on CPU: the cost
partition, and the per-rank solve + gather over a world-size-2 ``gloo`` process group with a
stand-in solve (no GPU).  A rank that fails before the gather ends the other rank's gather with
an error instead of a hang."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from realmolecule_b200 import shard


def clusters():
    rng = np.random.default_rng(3)
    return [{"NN": int(NN), "screen": NN * 0.25, "atoms": [], "tag": q}
            for q, NN in enumerate(rng.choice([48, 64, 80, 96, 112, 128], size=23))]


def test_partition_covers_every_instance_once_and_balances():
    inst = clusters()
    costs = [shard.instance_cost(i) for i in inst]
    for parts in (1, 2, 3, 8):
        p = shard.partition(costs, parts)
        assert len(p) == parts
        flat = sorted(q for part in p for q in part)
        assert flat == list(range(len(inst)))
        loads = [sum(costs[q] for q in part) for part in p]
        assert max(loads) - min(loads) <= max(costs)
        assert p == shard.partition(costs, parts)  # deterministic
        assert all(part == sorted(part) for part in p)


def test_partition_edge_cases():
    assert shard.partition([], 3) == [[], [], []]
    assert shard.partition([5.0], 2) == [[0], []]
    with pytest.raises(ValueError):
        shard.partition([1.0], 0)
    with pytest.raises(ValueError):
        shard.my_share(clusters(), 2, 2)


def fake_solve(share):
    """steps = 100 * tag, energy = -cost (a function of the instance alone)."""
    return (np.array([100 * i["tag"] for i in share], np.int32),
            np.array([-float(shard.instance_cost(i)) for i in share]))


def test_single_process_solves_everything():
    inst = clusters()
    conv, E = shard.solve_sharded(inst, fake_solve)
    ref_c, ref_E = fake_solve(inst)
    np.testing.assert_array_equal(conv, ref_c)
    np.testing.assert_array_equal(E, ref_E)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, fail_rank, q):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    inst = clusters()
    seen = []

    def solve(share):
        seen.extend(i["tag"] for i in share)
        if rank == fail_rank:
            raise RuntimeError("injected failure on this rank")
        return fake_solve(share)

    try:
        conv, E = shard.solve_sharded(inst, solve)
        q.put((rank, "ok", conv.tolist(), E.tolist(), seen))
    except Exception as e:  # noqa: BLE001 -- reported to the parent
        q.put((rank, "error", type(e).__name__, str(e)[:200], seen))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run(world, fail_rank):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, fail_rank, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    try:
        for _ in range(world):
            r = q.get(timeout=120)
            out[r[0]] = r[1:]
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    return out


def test_two_gloo_ranks_gather_the_same_results():
    out = _run(2, fail_rank=-1)
    inst = clusters()
    ref_c, ref_E = fake_solve(inst)
    for r in (0, 1):
        status, conv, E, seen = out[r]
        assert status == "ok"
        np.testing.assert_array_equal(conv, ref_c)
        np.testing.assert_array_equal(E, ref_E)
        assert sorted(seen) == sorted(inst[q]["tag"] for q in shard.my_share(inst, r, 2))
    assert not set(out[0][3]) & set(out[1][3])  # no instance solved twice


def test_failing_rank_ends_the_gather_with_an_error():
    out = _run(2, fail_rank=1)
    assert out[1][0] == "error" and "injected failure" in out[1][2]
    assert out[0][0] == "error"  # the surviving rank learns of it at the gather, no hang
