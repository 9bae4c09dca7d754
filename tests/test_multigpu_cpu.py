"""World-size-2 tests of the multi-GPU host logic on CPU (gloo): views sharded across
ranks, per-rank gradients (the oracle stands in for the device backward), one
all-reduce, compared with the single-process result; and a rank that fails before
the collective is seen by the other rank as an error, not a hang."""
import os
import socket
import traceback

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from ever_b200 import distributed as D
from ever_b200 import synthetic as S


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _scene():
    return S.uniform_scene(200, 1, seed=31)


def _views():
    return [S.Camera(S.sphere_point(3.0, 40 + i), 6, 5, 50.0) for i in range(3)]


def _view_grads(sc, cam):
    from oracle import oracle as O
    ro, rd = S.look_at_rays(cam)
    s = O.Scene(sc.mean, sc.scale, sc.quat, sc.density, sc.features)
    tr = O.trace(s, ro, rd, 0.0, 1000.0, 500, nthreads=1)
    dout = np.ones((ro.shape[0], 5))
    g = O.backward(s, ro, rd, 0.0, 1000.0, 500, tr.events, tr.iters, dout, nthreads=1)
    return [torch.tensor(x) for x in (g.mean, g.scale, g.quat, g.density, g.features)]


def _worker(rank, world, port, mode, result_dir):
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        from datetime import timedelta
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=20))
        sc = _scene()
        mine = D.view_shard(_views(), rank, world)
        if mode == "fail" and rank == 1:
            raise RuntimeError("injected host-side failure before the collective")
        grads = None
        for cam in mine:
            g = _view_grads(sc, cam)
            grads = g if grads is None else [a + b for a, b in zip(grads, g)]
        D.allreduce_gradients(grads)
        t = D.max_over_ranks(1.0 + rank, torch.device("cpu"))
        if rank == 0:
            torch.save({"grads": grads, "tmax": t}, os.path.join(result_dir, "rank0.pt"))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # recorded for the parent; never hangs the test
        with open(os.path.join(result_dir, f"err{rank}.txt"), "w") as f:
            f.write(f"{type(e).__name__}: {e}\n{traceback.format_exc()}")


def _bucket_worker(rank, world, port, result_dir):
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        from datetime import timedelta
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=20))
        calls = []
        real = dist.all_reduce

        def counting(t, *a, **k):
            calls.append(t.numel())
            return real(t, *a, **k)

        dist.all_reduce = counting
        g = torch.Generator().manual_seed(rank)
        ts = [torch.randn(5, 3, generator=g, dtype=torch.float64), None,
              torch.randn(5, 4, generator=g, dtype=torch.float64), torch.randn(5, generator=g, dtype=torch.float64)]
        D.allreduce_gradients(ts)
        dist.all_reduce = real
        if rank == 0:
            torch.save({"calls": calls, "ts": [t for t in ts if t is not None]}, os.path.join(result_dir, "b0.pt"))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:
        with open(os.path.join(result_dir, f"err{rank}.txt"), "w") as f:
            f.write(f"{type(e).__name__}: {e}\n{traceback.format_exc()}")


def test_one_bucketed_allreduce(tmp_path):
    port = _free_port()
    mp.start_processes(_bucket_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    assert not list(tmp_path.glob("err*.txt")), [p.read_text() for p in tmp_path.glob("err*.txt")]
    res = torch.load(tmp_path / "b0.pt")
    assert res["calls"] == [15 + 20 + 5]  # one collective over the packed bucket
    want = []
    for r in range(2):
        g = torch.Generator().manual_seed(r)
        want.append([torch.randn(5, 3, generator=g, dtype=torch.float64),
                     torch.randn(5, 4, generator=g, dtype=torch.float64), torch.randn(5, generator=g, dtype=torch.float64)])
    for got, a, b in zip(res["ts"], want[0], want[1]):
        torch.testing.assert_close(got, a + b)


def test_view_shard_round_robin():
    v = list(range(7))
    shards = [D.view_shard(v, r, 3) for r in range(3)]
    assert shards == [[0, 3, 6], [1, 4], [2, 5]]
    assert sorted(sum(shards, [])) == v
    with pytest.raises(ValueError):
        D.view_shard(v, 3, 3)


def test_sharded_gradients_match_single_process(tmp_path):
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, "ok", str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    assert not list(tmp_path.glob("err*.txt")), [p.read_text() for p in tmp_path.glob("err*.txt")]
    res = torch.load(tmp_path / "rank0.pt")
    sc = _scene()
    full = None
    for cam in _views():
        g = _view_grads(sc, cam)
        full = g if full is None else [a + b for a, b in zip(full, g)]
    for a, b in zip(res["grads"], full):
        np.testing.assert_allclose(a.numpy(), b.numpy(), rtol=1e-12, atol=1e-12)
    assert res["tmax"] == 2.0


def test_failed_rank_surfaces_as_error(tmp_path):
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, "fail", str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    errs = {p.name: p.read_text() for p in tmp_path.glob("err*.txt")}
    assert "err1.txt" in errs and "injected" in errs["err1.txt"]
    # rank 0 blocks in the all-reduce until the process-group timeout, then errors out
    assert "err0.txt" in errs, "surviving rank did not report the missing peer"
