"""Multi-GPU host logic (kerrtracecpp2_b200.shard) on the CPU: the tile
partition, the frame assignment, and -- as two gloo ranks on this host --
the gather of a tile-sharded frame and the all-reduce of a tile-sharded
gradient, with stand-in tracers (no GPU)."""
import os
import socket

import numpy as np
import pytest

from kerrtracecpp2_b200 import abi
from kerrtracecpp2_b200 import shard as S


@pytest.mark.parametrize("w,h,world,tile", [(100, 37, 3, 16), (1, 1, 2, 16), (7, 3, 4, 2),
                                            (1280, 720, 8, 16), (64, 64, 1, 8)])
def test_tiles_partition_the_frame(w, h, world, tile):
    parts = [S.frame_tiles(w, h, world, r, tile) for r in range(world)]
    allp = np.concatenate(parts)
    assert len(allp) == w * h and np.array_equal(np.sort(allp), np.arange(w * h))
    sizes = [len(p) for p in parts]
    assert max(sizes) - min(sizes) <= tile * tile


def test_assign_frames_balances_and_covers():
    rng = np.random.default_rng(0)
    costs = list(rng.uniform(1, 100, 64))
    parts = S.assign_frames(costs, 8)
    assert sorted(i for p in parts for i in p) == list(range(64))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) <= sum(costs) / 8 + max(costs)
    assert parts == S.assign_frames(costs, 8)


def test_frame_cost_follows_the_fallback_rules():
    ks = abi.frame_desc(chart=0, width=10, height=10)
    ks_lam = abi.frame_desc(chart=0, Lambda=1e-4, width=10, height=10)
    bl = abi.frame_desc(chart=1, width=10, height=10)
    ks_dopri = abi.frame_desc(chart=0, integrator=1, width=10, height=10)
    assert S.frame_cost(ks_lam) == S.frame_cost(bl) != S.frame_cost(ks)
    assert S.frame_cost(ks_dopri) == S.frame_cost(ks)


def _fake_trace(desc, pix):
    p = pix.astype(np.float64)
    return {"r": np.sqrt(p + 1.0), "outcome": (pix % 3).astype(np.uint8)}


def _fake_grad(desc, pix):
    p = pix.astype(np.float64)
    return float(np.sum(p * 1e-3)), [np.sum(np.sin(p)), np.sum(np.cos(p)), 0.0, np.sum(p % 7), 1.0 * len(p), 0.0]


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        d = abi.frame_desc(width=45, height=29)
        frame = S.trace_frame_sharded(None, d, trace=_fake_trace, tile=8)
        loss, grad = S.l2_grad_sharded(None, d, None, grad_fn=_fake_grad, tile=8)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), loss=loss, grad=grad,
                 has_frame=frame is not None,
                 **({f"f_{k}": v for k, v in frame.items()} if frame is not None else {}))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_frame_and_reduce_gradient(tmp_path):
    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.spawn(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    d = abi.frame_desc(width=45, height=29)
    n = d.width * d.height
    full = _fake_trace(d, np.arange(n, dtype=np.uint32))
    r0 = np.load(tmp_path / "rank0.npz")
    r1 = np.load(tmp_path / "rank1.npz")
    assert r0["has_frame"] and not r1["has_frame"]
    for k, v in full.items():
        assert np.array_equal(r0[f"f_{k}"], v)
    loss_full, grad_full = _fake_grad(d, np.arange(n, dtype=np.uint32))
    for r in (r0, r1):
        assert float(r["loss"]) == pytest.approx(loss_full, rel=1e-12)
        np.testing.assert_allclose(r["grad"], grad_full, rtol=1e-12, atol=1e-9)
