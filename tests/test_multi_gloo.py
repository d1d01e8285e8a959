"""The multi-rank path on CPU: world_size 2 over gloo (127.0.0.1).

Pairs are independent, so ranks only need a shared assignment, the max of
their step times and a gather of their records; the data path has no
collective.  Each rank also refines its own pairs with the FP64 oracle and
the gathered results must equal a single-process run."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    sys.path.insert(0, REPO)
    import torch.distributed as dist
    from datetime import timedelta
    import __graft_entry__
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    pkg = __graft_entry__.load_package()
    orc = __graft_entry__.load_oracle()
    orc.set_threads(1)
    sizes = [(80 + 7 * i) * (40 + 3 * i) for i in range(9)]
    mine = pkg.shard.shard(sizes, rank, world)
    recs = {}
    for i in mine:
        W, H = 80 + 7 * i, 40 + 3 * i
        pr = pkg.synth.make_pair(500 + i, W, H, 1.0, 12.0, n_planes=(1, 2))
        d0 = pr.disp.ravel() + np.random.default_rng(i).uniform(-2, 2, W * H)
        out, st = orc.lr_refine(pr.gray("left").ravel(), pr.gray("right").ravel(), d0, W, H,
                                tol=2.0, R=4, P1=12.0, P2=150.0, rx=2, ry=2)
        recs[i] = (float(out.sum()), int(st.sum()))
    t = pkg.shard.max_over_ranks(float(rank + 1))
    gathered = pkg.shard.gather_metrics({"rank": rank, "pairs": mine, "recs": recs})
    q.put((rank, t, gathered))
    dist.barrier()
    dist.destroy_process_group()


def test_shard_assignment_balanced_and_complete(svb):
    sizes = [1400 * 1100, 200 * 150, 640 * 480, 900 * 700, 300 * 300, 1000 * 1000, 256 * 192]
    parts = [svb.shard.shard(sizes, r, 3) for r in range(3)]
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(sizes)))
    loads = [sum(sizes[i] for i in p) for p in parts]
    assert max(loads) <= sum(sizes) / 3 + max(sizes)
    with pytest.raises(ValueError):
        svb.shard.shard(sizes, 3, 3)


def test_two_rank_gloo(svb, orc):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert [r[1] for r in res] == [2.0, 2.0]            # max over ranks
    gathered = res[0][2]
    assert gathered == res[1][2]
    pairs = sorted(i for g in gathered for i in g["pairs"])
    assert pairs == list(range(9))
    # the union of the ranks' results equals a single-process run
    allrecs = {int(k): v for g in gathered for k, v in g["recs"].items()}
    for i in (0, 4, 8):
        W, H = 80 + 7 * i, 40 + 3 * i
        pr = svb.synth.make_pair(500 + i, W, H, 1.0, 12.0, n_planes=(1, 2))
        d0 = pr.disp.ravel() + np.random.default_rng(i).uniform(-2, 2, W * H)
        out, st = orc.lr_refine(pr.gray("left").ravel(), pr.gray("right").ravel(), d0, W, H,
                                tol=2.0, R=4, P1=12.0, P2=150.0, rx=2, ry=2)
        assert allrecs[i] == (float(out.sum()), int(st.sum()))
