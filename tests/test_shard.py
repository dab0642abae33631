"""Multi-GPU host logic (kerrtracecpp2_b200.shard) on the CPU: the tile
partition, the frame assignment, and -- as two and three gloo ranks on this
host -- the gather of a tile-sharded frame and the all-reduce of a
tile-sharded gradient, with stand-in tracers (no GPU)."""
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


@pytest.mark.parametrize("w,h,world", [(1280, 720, 1), (1280, 720, 3), (45, 29, 2)])
def test_centre_out_tiles_are_the_same_pixels(w, h, world):
    """The centre-out order is a permutation of each rank's tile pixels,
    innermost ring first and row-major within a ring."""
    for r in range(world):
        a = S.frame_tiles(w, h, world, r, 16)
        b = S.frame_tiles(w, h, world, r, 16, centre_out=True)
        assert np.array_equal(np.sort(a), np.sort(b))
        x, y = (b % w).astype(float) - 0.5 * (w - 1), (b // w).astype(float) - 0.5 * (h - 1)
        ring = np.minimum((np.hypot(x, y) / max(4.0, (np.hypot(0.5 * (w - 1), 0.5 * (h - 1)) + 1) / 512)).astype(int), 511)
        assert np.all(np.diff(ring) >= 0)
        same = np.diff(ring) == 0
        assert np.all(np.diff(b.astype(np.int64))[same] > 0)


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


def _fake_grad(desc, pix):
    p = pix.astype(np.float64)
    return float(np.sum(p * 1e-3)), [np.sum(np.sin(p)), np.sum(np.cos(p)), 0.0, np.sum(p % 7), 1.0 * len(p), 0.0]


def _fake_trace_all_fields(desc, pix):
    """Every field of a kt_geo_soa with its dtype, values that use every bit
    pattern class (negative zero, NaN payloads, large counters)."""
    p = pix.astype(np.float64)
    r = np.sqrt(p + 1.0)
    r[pix % 11 == 0] = -0.0
    red = np.where(pix % 13 == 0, np.float64("nan"), 1.0 / (p + 3.0))
    return {"outcome": (pix % 3).astype(np.uint8), "r": r, "redshift": red, "magnif": p * 1e-300,
            "phi_disk": -p, "theta_esc": np.cos(p), "phi_esc": np.sin(p),
            "status": (pix % 5).astype(np.uint8),
            "steps": (pix * 2654435761).astype(np.uint32).view(np.int32),
            "attempts": (pix + 7).astype(np.int32)}


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        d = abi.frame_desc(width=45, height=29)
        frame = S.trace_frame_sharded(None, d, trace=_fake_trace_all_fields, tile=8)
        loss, grad = S.l2_grad_sharded(None, d, None, grad_fn=_fake_grad, tile=8)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), loss=loss, grad=grad,
                 has_frame=frame is not None,
                 **({f"f_{k}": v.numpy() for k, v in frame.items()} if frame is not None else {}))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_gather_frame_and_reduce_gradient(tmp_path, world):
    """2 and 3 gloo ranks: the tile-sharded frame arrives on rank 0 bit for
    bit (one byte-buffer gather of tensors, no pickling), and every rank
    gets the whole frame's loss and gradient from the all-reduce."""
    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.spawn(_worker, args=(world, port, str(tmp_path)), nprocs=world, join=True)
    d = abi.frame_desc(width=45, height=29)
    n = d.width * d.height
    full = _fake_trace_all_fields(d, np.arange(n, dtype=np.uint32))
    rs = [np.load(tmp_path / f"rank{q}.npz") for q in range(world)]
    assert rs[0]["has_frame"] and not any(r["has_frame"] for r in rs[1:])
    assert sorted(k[2:] for k in rs[0].files if k.startswith("f_")) == sorted(full)
    for k, v in full.items():
        got = rs[0][f"f_{k}"]
        assert got.dtype == v.dtype and got.tobytes() == v.tobytes(), k
    loss_full, grad_full = _fake_grad(d, np.arange(n, dtype=np.uint32))
    for r in rs:
        assert float(r["loss"]) == pytest.approx(loss_full, rel=1e-12)
        np.testing.assert_allclose(r["grad"], grad_full, rtol=1e-12, atol=1e-9)
