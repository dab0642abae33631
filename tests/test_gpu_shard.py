"""The tile split on the GPU (kerrtracecpp2_b200.shard) through NCCL, as one
rank: every field of the gathered frame equals kt_trace's bit for bit, and
the sharded gradient's all-reduce gives kt_l2_grad's.  (Runs with more
ranks use the same calls; this box has one GPU.)"""
import os
import socket

import numpy as np
import pytest

from kerrtracecpp2_b200 import abi

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nccl_group():
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    if dist.is_initialized():
        yield None
        return
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=timedelta(seconds=120))
    yield None
    dist.destroy_process_group()


@pytest.mark.parametrize("kw", [
    dict(chart=1, integrator=1, tol=1e-10, a=0.9, Q=0.3, Lambda=1e-4, r_obs=60.0, theta_deg=85.0,
         fov_deg=30.0, disk_out=20.0, width=320, height=180),
    dict(chart=0, a=0.7, Q=0.1, theta_deg=70.0, r_obs=50.0, disk_out=15.0, width=200, height=120),
], ids=["bl_dopri5", "ks_rk4"])
def test_tile_sharded_frame_equals_kt_trace(renderer, nccl_group, kw):
    import torch

    from kerrtracecpp2_b200 import shard

    d = abi.frame_desc(**kw)
    whole = renderer.trace(d)
    torch.cuda.synchronize()
    frame = shard.trace_frame_sharded(renderer, d)
    torch.cuda.synchronize()
    assert frame is not None
    for k, v in whole.items():
        if v is None:
            continue
        a = frame[k].cpu().numpy()
        b = v.cpu().numpy()
        assert a.dtype == b.dtype and a.tobytes() == b.tobytes(), k


def test_tile_sharded_gradient_equals_whole_frame(renderer, nccl_group):
    from kerrtracecpp2_b200 import shard

    base = dict(chart=0, a=0.7, Q=0.1, Lambda=0.0, theta_deg=70.0, r_obs=50.0, disk_out=15.0,
                width=128, height=96)
    tgt = renderer.trace(abi.frame_desc(precision=abi.KT_PREC_SMOOTH, **dict(base, a=0.72, theta_deg=71.0)))
    d = abi.frame_desc(**base)
    loss, grad, _ = renderer.l2_grad(d, tgt, 1.0, 0.01)
    loss_s, grad_s = shard.l2_grad_sharded(renderer, d, tgt, 1.0, 0.01)
    assert loss_s == pytest.approx(loss, rel=1e-12)
    np.testing.assert_allclose(grad_s, grad, rtol=1e-10, atol=1e-12 * np.abs(grad).max())
