"""Helpers of the boundary tests: .kgeo files as the reference reads them,
binary PPM backgrounds for the CLI, and the reference's spin-orientation
analysis."""
import numpy as np

import oracle_lib as O


def kgeo_records(path):
    """-> (W, H, the 10 header doubles, GeoPixel records) of a .kgeo file
    (main.cpp:96-137: magic, version 1, KGeoMeta, 28-byte GeoPixel)."""
    raw = open(path, "rb").read()
    assert raw[:4] == b"KGEO" and np.frombuffer(raw[4:8], "<u4")[0] == 1
    W, H = (int(x) for x in np.frombuffer(raw[8:16], "<u4"))
    meta = np.frombuffer(raw[16:96], "<f8")
    assert len(raw) == 96 + 28 * W * H
    return W, H, meta, np.frombuffer(raw[96:], O.GEOPIXEL_DTYPE)


def write_ppm(path, img):
    with open(path, "wb") as f:
        f.write(b"P6\n%d %d\n255\n" % (img.shape[1], img.shape[0]))
        f.write(np.ascontiguousarray(img, np.uint8).tobytes())


def orientation(recs, W, H):
    """analyze_orientation of the reference's spin regression
    (tests/spin_orientation_regression.cpp:107-176), on GeoPixel records with
    their 28-byte stride: whether the hottest disk pixels (redshift at or
    above the 97th percentile, linear interpolation) lie right of the shadow's
    centroid, and whether the column with the largest gap above the shadow
    between the first disk pixel and the first horizon pixel does."""
    out = recs["outcome"].reshape(H, W)
    red = recs["redshift"].reshape(H, W)
    ys, xs = np.nonzero(out == 2)
    assert xs.size
    cx, cy = xs.astype(np.float64).mean(), ys.astype(np.float64).mean()
    disk = (out == 1) & np.isfinite(red)
    v = np.sort(red[disk].astype(np.float64))
    t = 0.97 * (v.size - 1)
    i0, i1 = int(np.floor(t)), int(np.ceil(t))
    q97 = v[i0] if i0 == i1 else v[i0] + (t - i0) * (v[i1] - v[i0])
    hot = disk & (red.astype(np.float64) >= q97)
    hot_x = np.nonzero(hot)[1].astype(np.float64).mean()
    y_top = max(1, int(np.floor(cy)))
    best_gap, best_x = -1, -1
    for x in range(W):
        col = out[:y_top, x]
        yh = np.nonzero(col == 2)[0]
        yd = np.nonzero(col == 1)[0]
        if yh.size == 0 or yd.size == 0:
            continue
        gap = int(yh[0]) - int(yd[0])
        if gap > best_gap:
            best_gap, best_x = gap, x
    assert best_x >= 0
    return hot_x > cx, best_x > cx
