"""Multi-rank logic on CPU (gloo, world size 2): shot sharding and the single
image reduction give the same Born adjoint image as one process over all shots
(CPU oracle as the per-rank engine, small grid); a rank that fails is reported
to the caller instead of hanging the others."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from acoustic_isotropic_operators_b200.multigpu import shard


def test_shard_covers_every_shot_once():
    for n in (1, 5, 32, 33):
        for w in (1, 2, 3, 8):
            got = [i for r in range(w) for i in shard(n, r, w)]
            assert got == list(range(n))
    with pytest.raises(ValueError):
        shard(4, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out, fail_rank):
    import sys
    import torch
    import torch.distributed as dist
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.join(os.path.dirname(here), "oracle"))
    import orc
    from cases import make_case
    from acoustic_isotropic_operators_b200.multigpu import max_over_ranks, reduce_image, shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        if rank == fail_rank:
            raise RuntimeError("injected failure on rank %d" % rank)
        c = make_case(seed=2, nzi=24, nxi=32, nts=20, sub=2, nshots=3)
        d = [np.random.default_rng(10 + i).standard_normal((len(c.rec_pos[i]), c.scheme.nts)) for i in range(3)]
        img = np.zeros((c.nx, c.nz))
        for i in shard(3, rank, world):
            img += orc.born_adj(c.scheme, c.vel, d[i], c.sig[i], c.src_pos[i], c.rec_pos[i])
        t = torch.from_numpy(img)
        reduce_image(t)
        slowest = max_over_ranks(float(rank + 1))
        if rank == 0:
            ref = sum(orc.born_adj(c.scheme, c.vel, d[i], c.sig[i], c.src_pos[i], c.rec_pos[i]) for i in range(3))
            out.put(("ok", float(np.linalg.norm(t.numpy() - ref) / np.linalg.norm(ref)), slowest))
    except Exception as e:  # reported to the parent; the other rank's collective times out
        out.put(("error", rank, str(e)))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run(world, fail_rank):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, fail_rank)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
    res = []
    while not q.empty():
        res.append(q.get())
    return res


def test_sharded_image_equals_single_process():
    res = _run(2, fail_rank=-1)
    ok = [r for r in res if r[0] == "ok"]
    assert ok and ok[0][1] < 1e-12, res
    assert ok[0][2] == 2.0      # max over ranks


def test_failed_rank_is_reported():
    res = _run(2, fail_rank=1)
    errs = [r for r in res if r[0] == "error"]
    assert any(r[1] == 1 and "injected" in r[2] for r in errs), res
