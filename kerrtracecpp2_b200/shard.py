"""Splitting the path across GPUs (one process per GPU, torch.distributed).

Rays are independent, so a frame, a batch of frames or a gradient divides
across ranks with no exchange on the data path; the only collective is the
gradient's one all-reduce of its few doubles:

  frame_tiles(W, H, world, rank, tile)   square tiles of the frame dealt
                                         round-robin: rank's pixel indices
  assign_frames(costs, world)            longest-first greedy assignment of
                                         a batch's frames by estimated cost
  frame_cost(desc)                       that estimate: W*H times a
                                         per-chart/integrator step prior
  trace_frame_sharded(renderer, desc, group)
                                         each rank traces its tiles
                                         (kt_trace_pixels), rank 0 gathers
                                         the frame (one byte-buffer gather
                                         of tensors, NCCL on the GPU)
  l2_grad_sharded(renderer, desc, target, w_g, w_r, group)
                                         each rank the gradient of its tiles
                                         (kt_l2_grad_pixels), one all-reduce

Interleaved tiles balance the very uneven cost of rays (a frame's step
counts differ by 3-50x between the sky, the disk and the critical curve)
better than contiguous bands.  The functions that move data take an
optional `trace` callable so the host logic runs without a GPU in tests.
"""
import numpy as np

from . import abi


def frame_tiles(width, height, world, rank, tile=16, centre_out=False):
    """Pixel indices (py*width + px, uint32, ascending within each tile) of
    the tiles of side `tile` dealt to `rank`: tile k goes to rank k % world,
    tiles numbered row-major.  With centre_out, the same pixels in the
    renderer's centre-out order (rings 4 pixels wide about the image centre,
    innermost first, row-major within a ring), so that each rank's longest
    rays -- by the critical curve, near the centre -- start first."""
    if not (0 <= rank < world):
        raise ValueError("rank out of range")
    tx = (width + tile - 1) // tile
    ty = (height + tile - 1) // tile
    out = []
    for k in range(rank, tx * ty, world):
        y0, x0 = (k // tx) * tile, (k % tx) * tile
        ys = np.arange(y0, min(y0 + tile, height), dtype=np.int64)
        xs = np.arange(x0, min(x0 + tile, width), dtype=np.int64)
        out.append((ys[:, None] * width + xs[None, :]).ravel())
    if not out:
        return np.zeros(0, np.uint32)
    pix = np.concatenate(out)
    if centre_out:
        pix = np.sort(pix)
        cx, cy = np.float32(0.5 * (width - 1)), np.float32(0.5 * (height - 1))
        rmax = np.sqrt(cx * cx + cy * cy) + np.float32(1.0)
        inv_w = np.float32(1.0) / np.maximum(np.float32(4.0), rmax / np.float32(512))
        dx = (pix % width).astype(np.float32) - cx
        dy = (pix // width).astype(np.float32) - cy
        ring = np.minimum((np.sqrt(dx * dx + dy * dy) * inv_w).astype(np.int64), 511)
        pix = pix[np.argsort(ring, kind="stable")]
    return pix.astype(np.uint32)


# Mean adaptive attempts per ray measured on the benchmark frames, by
# (chart, integrator, bundles): a prior for balancing, not a promise.
_STEP_PRIOR = {(0, 0, 0): 65.0, (1, 0, 0): 90.0, (1, 1, 0): 145.0, (1, 0, 1): 600.0}


def frame_cost(desc):
    """Estimated cost of a frame: W*H times the prior attempts per ray of its
    effective chart/integrator (KS+Lambda and bundles run in BL, the KS chart
    ignores DOPRI5)."""
    chart = desc.chart
    if chart == abi.KT_CHART_KS and (abs(desc.Lambda) > 1e-15 or desc.bundles):
        chart = abi.KT_CHART_BL
    intg = desc.integrator if chart == abi.KT_CHART_BL else abi.KT_RK4_DOUBLING
    prior = _STEP_PRIOR.get((chart, intg, int(bool(desc.bundles))), 100.0)
    return float(desc.width) * float(desc.height) * prior


def assign_frames(costs, world):
    """Longest-processing-time greedy: frames in decreasing cost, each to the
    least-loaded rank (ties to the lower rank).  Returns a list of frame
    index lists, one per rank, each in increasing order; deterministic."""
    loads = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        r = min(range(world), key=lambda q: (loads[q], q))
        loads[r] += costs[i]
        parts[r].append(i)
    return [sorted(p) for p in parts]


def _dist():
    import torch.distributed as dist

    return dist


_PLANS = {}


def _plan(width, height, world, tile, centre_out, device):
    """Every rank's tile pixels (host) and their device index tensors for a
    frame shape, built once per (shape, world, tile, order, device)."""
    import torch

    key = (width, height, world, tile, centre_out, str(device))
    if key not in _PLANS:
        parts = [frame_tiles(width, height, world, q, tile, centre_out) for q in range(world)]
        _PLANS[key] = (parts,
                       [torch.from_numpy(p.astype(np.int32)).to(device) for p in parts],
                       [torch.from_numpy(p.astype(np.int64)).to(device) for p in parts])
    return _PLANS[key]


def _as_tensor(v, device):
    import torch

    if isinstance(v, torch.Tensor):
        return v.to(device).contiguous()
    return torch.from_numpy(np.ascontiguousarray(v)).to(device)


def trace_frame_sharded(renderer, desc, group=None, tile=16, trace=None, dst=0, fields=None,
                        centre_out=True):
    """Trace one frame split over the ranks of `group` by tiles.  Every rank
    traces its own tiles (kt_trace_pixels on its GPU, or `trace(desc, pix)`
    returning a dict of arrays or tensors per pixel); the parts travel to
    rank `dst` as one byte buffer per rank (each field's bytes, padded to
    the largest part) in a single gather -- over NCCL for device tensors,
    gloo for host ones -- and are scattered into the frame there.  Rank
    `dst` returns the whole frame as a dict of tensors on the parts' device,
    bit for bit what each rank traced; the other ranks return None.
    `fields` (default: every field the trace returned) chooses what
    travels; each rank traces its pixels in centre-out order unless
    centre_out is False (the results do not depend on the order)."""
    import torch

    dist = _dist()
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    dev = torch.device("cuda", renderer.device) if trace is None else torch.device("cpu")
    parts, pix32, idx64 = _plan(desc.width, desc.height, world, tile, centre_out, dev)
    pix = parts[rank]
    res = renderer.trace_pixels(desc, pix32[rank]) if trace is None else trace(desc, pix)
    keys = sorted(k for k, v in res.items() if v is not None and (fields is None or k in fields))
    vals = {k: _as_tensor(res[k], dev) for k in keys}
    m = max(len(p) for p in parts)
    sizes = {k: vals[k].element_size() for k in keys}
    row = sum(sizes.values())
    buf = torch.zeros(m * row, dtype=torch.uint8, device=dev)
    off = 0
    for k in keys:
        nb = len(pix) * sizes[k]
        buf[off:off + nb] = vals[k].view(torch.uint8)
        off += m * sizes[k]
    gathered = [torch.empty_like(buf) for _ in range(world)] if rank == dst else None
    dist.gather(buf, gathered, dst=dst, group=group)
    if rank != dst:
        return None
    n = desc.width * desc.height
    frame = {k: torch.zeros(n, dtype=vals[k].dtype, device=dev) for k in keys}
    for q in range(world):
        idx = idx64[q]
        off = 0
        for k in keys:
            nb = len(parts[q]) * sizes[k]
            frame[k][idx] = gathered[q][off:off + nb].view(vals[k].dtype)
            off += m * sizes[k]
    return frame


def l2_grad_sharded(renderer, desc, target, w_g=1.0, w_r=0.0, group=None, tile=16, grad_fn=None):
    """Gradient of the L2 image loss of one frame split over the ranks of
    `group`: each rank the loss and gradient of its tiles
    (kt_l2_grad_pixels, or `grad_fn(desc, pix)` returning (loss, grad)),
    then one all-reduce (sum) of [loss, grad...].  Every rank returns
    (loss, grad)."""
    import torch

    dist = _dist()
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    pix = frame_tiles(desc.width, desc.height, world, rank, tile)
    if grad_fn is None:
        dev = torch.device("cuda", renderer.device)
        loss, grad, _ = renderer.l2_grad(desc, target, w_g, w_r,
                                         pix=torch.from_numpy(pix.astype(np.int32)).to(dev))
        buf = torch.tensor([loss] + list(grad), dtype=torch.float64, device=dev)
    else:
        loss, grad = grad_fn(desc, pix)
        buf = torch.tensor([loss] + list(grad), dtype=torch.float64)
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    out = buf.cpu().numpy()
    return float(out[0]), out[1:]
