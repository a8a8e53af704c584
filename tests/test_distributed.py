"""The kNN split across ranks (umappp_b200.distributed), on CPUs: two gloo
ranks, each computing its shard with the oracle's exact search (standing in for
umapb_knn_shard, which needs a GPU) over rows of its own, then one all-gather;
both ranks must end with the oracle's full lists.  Shards of unequal size and
a rank with no rows are covered; ranks whose rows overlap are rejected; a rank
whose search raises makes every rank raise (none waits in the gather); and
initialize_sharded hands the full lists to the rest of the pipeline (a
stand-in for initialize_knn_matrix) on every rank."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n, k, mode, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import oracle
    from umappp_b200.distributed import initialize_sharded, knn_sharded

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        X = oracle.gaussian_mixture(n, 5, 3, 3.0, seed=5, dtype=np.float32)

        def local(x, kk, r, w):
            if mode == "fail" and r == 1:
                raise ValueError("stand-in search failure")
            if mode in ("uneven", "init"):   # rank 0 takes a third, rank 1 the rest
                lo, hi = (0, n // 3) if r == 0 else (n // 3, n)
            elif mode == "empty":      # rank 0 takes nothing
                lo, hi = (0, 0) if r == 0 else (0, n)
            else:                      # overlapping rows: must be rejected
                lo, hi = (0, n // 2 + 5) if r == 0 else (n // 2, n)
            rows = np.arange(lo, hi, dtype=np.int32)
            idx, d = oracle.knn(x, kk, lo, hi - lo) if hi > lo else (np.zeros((0, kk), np.int32), np.zeros((0, kk)))
            return rows, idx, d.astype(np.float32)

        try:
            ridx, rd = oracle.knn(X, k)
            if mode == "init":
                # the rest of the pipeline gets the full lists on every rank
                from umappp_b200 import Options

                def init(i, dd, num_dim, emb, opt):
                    return ("status", bool(np.array_equal(i, ridx) and np.array_equal(dd, rd.astype(np.float32))),
                            num_dim, emb.shape, opt.num_neighbors)

                got = initialize_sharded(X, 2, np.zeros((n, 2), np.float32), Options(num_neighbors=k),
                                         local=local, init=init)
                q.put((rank, "ok", got == ("status", True, 2, (n, 2), k)))
            else:
                idx, d = knn_sharded(X, k, local=local)
                q.put((rank, "ok", bool(np.array_equal(idx, ridx) and np.array_equal(d, rd.astype(np.float32)))))
        except (RuntimeError, ValueError) as e:
            q.put((rank, "error", str(e)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("mode", ["uneven", "empty", "overlap", "fail", "init"])
def test_knn_sharded_gather_two_ranks(mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, 301, 7, mode, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs)
    if mode == "overlap":
        assert all(r[1] == "error" and "partition" in r[2] for r in results), results
    elif mode == "fail":   # every rank raises: rank 1 its own error, rank 0 that another rank failed
        results = sorted(results)
        assert [r[1] for r in results] == ["error", "error"], results
        assert "another rank" in results[0][2] and "stand-in search failure" in results[1][2], results
    else:
        assert all(r[1] == "ok" and r[2] for r in results), results
