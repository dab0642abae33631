"""Central-difference check of a gradient on the GPU (shared by
tests/test_gpu_grad.py and bench.py's adjoint leg).

The default frame (config 5): 512x512 KS, a=0.7, Q=0.1, theta=70, r_obs=50,
disk ISCO-15, tol 1e-7; the loss: sum over the disk pixels of both frames of
w_g (g - g_t)^2 + w_r (r_hit - r_t)^2 against the smooth tracer at a=0.72,
theta=71.  CFG2_DOPRI5 (the DOPRI5 adjoint) and BUNDLE (the Jacobi-bundle
adjoint, its loss with w_m (magnif - magnif_t)^2 as well) use the same
check.  The adjoint (kt_vjp with the loss's cotangents) is compared with
central differences of the same loss, restricted to the pixels on which the
stencil renders lie on one smooth piece of the point-sampled image (a pixel
that changes class, step or attempt count is a discontinuity of the image,
not of the integrator's derivative):

  five-point, h = 1e-4 (theta in radians; Lambda 1e-6): renders at +-h, +-2h;
      a pixel also needs small second differences of g and r_hit and central
      differences over h and 2h that agree to 1e-4 (no kink);
  two-point, h = 1e-6 (Lambda 1e-8): renders at +-h, on the five-point
      check's smooth pixels that keep class, step and attempt counts at +-h
      ("two_point"), and on every pixel that keeps them ("two_point_loose").

At h = 1e-6 the differences divide the renders' own rounding noise by 2h:
about 1e-13 in the median pixel's g and 2e-11 at p99 (the smooth tracer
forms its error estimate from the paths' increments; from the end states it
was 2e-12 and 8e-10), plus a few pixels whose g jumps at that scale with
their step sequence unchanged, which only the loose mask keeps.
"""
import numpy as np

from kerrtracecpp2_b200 import abi

CFG5 = dict(chart=0, a=0.7, Q=0.1, Lambda=0.0, theta_deg=70.0, r_obs=50.0, disk_out=15.0,
            width=512, height=512)
W_G, W_R = 1.0, 0.01
PARAMS = ("a", "Q", "Lambda", "theta_deg", "r_obs")


def _np(out):
    import torch

    torch.cuda.synchronize()
    got = {k: (v.cpu().numpy() if v is not None else None) for k, v in out.items()}
    got["steps"] = got["steps"].view(np.uint32)
    got["attempts"] = got["attempts"].view(np.uint32)
    return got


# Configuration 2's geometry with DOPRI5 at tol 1e-10 (the BL DOPRI5 adjoint),
# its loss against the same tracer at a=0.92, theta=86.
CFG2_DOPRI5 = dict(chart=1, integrator=1, tol=1e-10, a=0.9, Q=0.3, Lambda=1e-4, r_obs=60.0,
                   theta_deg=85.0, fov_deg=30.0, disk_out=20.0, width=320, height=180)
TARGET_CFG2 = dict(a=0.92, theta_deg=86.0)

# A KNdS Jacobi-bundle frame (BL, RK4 step doubling, tol 1e-9) for the
# bundle adjoint, its loss with the magnification (weight W_M) against the
# same tracer at a=0.92, theta=71.
BUNDLE = dict(chart=1, bundles=1, a=0.9, Q=0.2, Lambda=1e-5, theta_deg=70.0, r_obs=40.0,
              fov_deg=30.0, disk_out=12.0, tol=1e-9, max_steps=20000, width=320, height=180)
TARGET_BUNDLE = dict(a=0.92, theta_deg=71.0)
W_M = 0.01


def fd_check(renderer, base=CFG5, h4=1e-4, h2=1e-6, target=None, w_m=0.0):
    """Returns {"five_point": .., "two_point": .., "two_point_loose": ..},
    each with the per-parameter adjoint, difference and relative
    disagreement, the worst of them and the number of pixels in the loss.
    With w_m, the loss also holds w_m (magnif - magnif_t)^2 (bundles)."""
    import torch

    def smooth(kw):
        return _np(renderer.trace(abi.frame_desc(precision=abi.KT_PREC_SMOOTH, **kw)))

    tgt = smooth(dict(base, **(target or dict(a=0.72, theta_deg=71.0))))
    b0 = smooth(base)
    bl0 = b0 if base.get("chart", 0) == 1 else smooth(dict(base, chart=1))
    m_all = (b0["outcome"] == 1) & (tgt["outcome"] == 1)
    fields = ("redshift", "r", "magnif") if w_m else ("redshift", "r")

    def loss_on(o, ok):
        L = np.sum(W_G * (o["redshift"][ok] - tgt["redshift"][ok]) ** 2 +
                   W_R * (o["r"][ok] - tgt["r"][ok]) ** 2)
        if w_m:
            L += np.sum(w_m * (o["magnif"][ok] - tgt["magnif"][ok]) ** 2)
        return L

    def adjoint(ok):
        def cot(o):
            c = (torch.from_numpy(np.where(ok, 2 * W_G * (o["redshift"] - tgt["redshift"]), 0.0)).cuda(),
                 torch.from_numpy(np.where(ok, 2 * W_R * (o["r"] - tgt["r"]), 0.0)).cuda())
            m = (torch.from_numpy(np.where(ok, 2 * w_m * (o["magnif"] - tgt["magnif"]), 0.0)).cuda()
                 if w_m else None)
            return c, m

        (cg, cr), cm = cot(b0)
        if base.get("chart", 0) == 1:  # BL: Lambda from the same reverse sweep
            g, _ = renderer.vjp(abi.frame_desc(**base), cg, cr, cot_magnif=cm)
            gl = g
        else:
            g, _ = renderer.vjp(abi.frame_desc(**base), cg, cr, flags=abi.KT_GRAD_SKIP_LAMBDA)
            gl, _ = renderer.vjp(abi.frame_desc(**dict(base, chart=1)), *cot(bl0)[0])
        return {"a": g[0], "Q": g[1], "Lambda": gl[2], "theta_deg": g[3], "r_obs": g[4]}

    def stencil(k, hk, js):
        return {j: smooth(dict(base, **{k: base[k] + j * hk})) for j in js}

    def same_piece(o0, o, ok):
        ok &= (o0["outcome"] == 1) & (o["outcome"] == 1)
        for f in ("steps", "attempts"):
            ok &= o[f] == o0[f]
        return ok

    # five-point, h4
    ok = m_all.copy()
    renders = {}
    for k in PARAMS:
        hk = 1e-6 if k == "Lambda" else (np.degrees(h4) if k == "theta_deg" else h4)
        o0 = bl0 if k == "Lambda" else b0
        rs = stencil(k, hk, (-2, -1, 1, 2))
        renders[k] = (rs, hk)
        for o in rs.values():
            ok = same_piece(o0, o, ok)
        for f in fields:
            for j in (1, 2):
                op, om = rs[j][f], rs[-j][f]
                ok &= np.abs(op - 2 * o0[f] + om) <= 1e-8 + 0.01 * np.abs(op - om)
            d1, d2 = rs[1][f] - rs[-1][f], rs[2][f] - rs[-2][f]
            ok &= np.abs(d2 - 2 * d1) <= 1e-12 + 1e-4 * np.abs(d1)
    adj = adjoint(ok)
    five = {"h": h4, "pixels": int(ok.sum()), "disk_pixels": int(m_all.sum()), "per_param": {}}
    for k, (rs, hk) in renders.items():
        L = {j: loss_on(o, ok) for j, o in rs.items()}
        fd4 = (L[-2] - 8 * L[-1] + 8 * L[1] - L[2]) / (12 * hk)
        five["per_param"][k] = {"adjoint": adj[k], "fd": fd4, "rel": abs(adj[k] - fd4) / abs(fd4)}
    five["worst_rel"] = max(v["rel"] for v in five["per_param"].values())

    # two-point, h2: on the five-point check's smooth pixels (whose stencil
    # over [-2 h4, 2 h4] contains this one) that keep class and step sequence
    # at +-h2, and on every pixel that keeps them at +-h2 (loose)
    ok2 = m_all.copy()
    renders2 = {}
    for k in PARAMS:
        hk = h2 * 1e-2 if k == "Lambda" else (np.degrees(h2) if k == "theta_deg" else h2)
        o0 = bl0 if k == "Lambda" else b0
        rs = stencil(k, hk, (-1, 1))
        renders2[k] = (rs, hk)
        for o in rs.values():
            ok2 = same_piece(o0, o, ok2)
    out = {"five_point": five}
    for name, mask in (("two_point", ok2 & ok), ("two_point_loose", ok2)):
        adj2 = adjoint(mask)
        two = {"h": h2, "pixels": int(mask.sum()), "disk_pixels": int(m_all.sum()), "per_param": {}}
        for k, (rs, hk) in renders2.items():
            fd2 = (loss_on(rs[1], mask) - loss_on(rs[-1], mask)) / (2 * hk)
            two["per_param"][k] = {"adjoint": adj2[k], "fd": fd2, "rel": abs(adj2[k] - fd2) / abs(fd2)}
        two["worst_rel"] = max(v["rel"] for v in two["per_param"].values())
        out[name] = two
    return out
