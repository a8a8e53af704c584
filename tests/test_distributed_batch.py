"""A batch of independent runs split across ranks (umappp_b200.distributed),
on CPUs.  partition_instances is checked directly (a partition, balanced to
within the largest instance, the same for the same input).  batch_sharded is
run by gloo ranks with a stand-in for batch_run (which needs a GPU) that
writes a layout depending on each instance's own rows and size, so that a
wrong instance boundary, a wrong write-back or a wrong gather shows up; every
rank must end with the layouts the stand-in gives on the whole batch at once.
Covered: numpy and torch arrays, without the gather (only the rank's own
instances written), more ranks than instances, and a rank whose run raises
(every rank raises, none waits)."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from umappp_b200.distributed import partition_instances  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _stand_in(data, sizes, num_dim, embedding, options, fail=False):
    """Layout of each instance: column 0 its rows' first coordinate, column 1
    its own mean of the second coordinate plus its size (so that instance
    boundaries matter)."""
    if fail:
        raise ValueError("stand-in failure")
    is_np = isinstance(data, np.ndarray)
    d = data if is_np else data.numpy()
    out = np.zeros((d.shape[0], num_dim), dtype=d.dtype)
    pos = 0
    for m in np.asarray(sizes, dtype=np.int64):
        m = int(m)
        blk = d[pos:pos + m]
        out[pos:pos + m, 0] = blk[:, 0]
        out[pos:pos + m, 1] = blk[:, 1].mean() + m if m else 0
        pos += m
    if is_np:
        embedding[:] = out
    else:
        embedding.copy_(torch.from_numpy(out))
    return {"sgd": float(len(sizes))}


def _batch(seed=3):
    rng = np.random.default_rng(seed)
    sizes = rng.integers(5, 60, size=9)
    X = rng.standard_normal((int(sizes.sum()), 4)).astype(np.float32)
    return sizes, X


def _worker(rank, world, port, mode, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    from umappp_b200.distributed import batch_sharded

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sizes, X = _batch()
        if mode == "few":
            sizes, X = sizes[:2], X[:int(sizes[:2].sum())]
        n = X.shape[0]
        expect = np.zeros((n, 2), np.float32)
        _stand_in(X, sizes, 2, expect, None)
        emb = np.full((n, 2), -7.0, np.float32)
        data = X
        if mode == "torch":
            data, emb = torch.from_numpy(X), torch.from_numpy(emb)

        def run(d, s, nd, e, o):
            return _stand_in(d, s, nd, e, o, fail=(mode == "fail" and rank == 1))

        try:
            out = batch_sharded(data, sizes, 2, emb, None, run=run, gather=(mode != "nogather"))
        except Exception as e:  # noqa: BLE001
            q.put((rank, "error", type(e).__name__ + ": " + str(e)))
            return
        e_np = emb.numpy() if mode == "torch" else emb
        offs = np.concatenate([[0], np.cumsum(sizes)])
        if mode == "nogather":
            mine = np.zeros(n, bool)
            for i in out["instances"]:
                mine[offs[i]:offs[i + 1]] = True
            ok = bool(np.array_equal(e_np[mine], expect[mine]) and np.all(e_np[~mine] == -7.0))
        else:
            ok = bool(np.array_equal(e_np, expect))
        q.put((rank, "ok", ok, [int(i) for i in out["instances"]]))
    finally:
        dist.destroy_process_group()


def _run(world, mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, mode, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    return results


def test_partition_instances():
    rng = np.random.default_rng(11)
    for world in (1, 2, 3, 8, 70):
        sizes = rng.integers(0, 50_000, size=64)
        parts = partition_instances(sizes, world)
        assert len(parts) == world
        allp = np.sort(np.concatenate(parts))
        assert np.array_equal(allp, np.arange(len(sizes)))
        assert all(np.all(np.diff(p) > 0) for p in parts)
        loads = np.array([sizes[p].sum() for p in parts])
        if world <= len(sizes):
            assert loads.max() - loads.min() <= sizes.max()
        for a, b in zip(parts, partition_instances(sizes, world)):
            assert np.array_equal(a, b)
    with pytest.raises(ValueError):
        partition_instances([3, -1], 2)
    with pytest.raises(ValueError):
        partition_instances([3], 0)


@pytest.mark.parametrize("mode", ["numpy", "torch", "nogather"])
def test_batch_sharded_two_ranks(mode):
    results = _run(2, mode)
    assert all(r[1] == "ok" and r[2] for r in results), results
    got = sorted(i for r in results for i in r[3])
    assert got == list(range(9))


def test_batch_sharded_more_ranks_than_instances():
    results = _run(3, "few")
    assert all(r[1] == "ok" and r[2] for r in results), results
    assert sorted(len(r[3]) for r in results) == [0, 1, 1]


def test_batch_sharded_failure_reaches_every_rank():
    results = _run(2, "fail")
    assert [r[1] for r in results] == ["error", "error"], results
    assert "stand-in failure" in results[1][2]
    assert "another rank" in results[0][2]
