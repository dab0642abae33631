"""Access to tests/golden/frames.npz (fixtures made by make_golden.py from
the reference renderer compiled here)."""
import json
import os

import numpy as np

from kerrtracecpp2_b200 import abi

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "frames.npz")
FIELDS = ("outcome", "r", "redshift", "magnif", "phi_disk", "theta_esc", "phi_esc")
_z = None


def data():
    global _z
    if _z is None:
        _z = dict(np.load(PATH))
    return _z


def cases():
    return json.loads(bytes(data()["meta_json"]).decode())


def desc(name):
    return abi.frame_desc(**cases()[name])


def result(name):
    z = data()
    return {k: z[f"{name}/{k}"] for k in FIELDS}


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view({1: np.uint8, 4: np.uint32, 8: np.uint64}[a.dtype.itemsize])


def mismatches(got, want, fields=FIELDS):
    """Per-field count of entries whose bits differ."""
    return {k: int(np.sum(bits(np.asarray(got[k], dtype=want[k].dtype)) != bits(want[k])))
            for k in fields}


COLOUR_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "colour.npz")
_zc = None


def colour():
    """tests/golden/colour.npz (make_colour_golden.py): interstellar palette
    images and camera_spp renders from the reference."""
    global _zc
    if _zc is None:
        _zc = dict(np.load(COLOUR_PATH))
    return _zc


def colour_meta():
    return json.loads(bytes(colour()["meta_json"]).decode())


SEMI_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "semi.npz")
_zs = None


def semi():
    """tests/golden/semi.npz (make_semi_golden.py): the semi-analytic solver."""
    global _zs
    if _zs is None:
        _zs = dict(np.load(SEMI_PATH))
    return _zs


def semi_cases():
    return json.loads(bytes(semi()["meta_json"]).decode())


def semi_desc(name):
    return abi.frame_desc(**semi_cases()[name])


def semi_result(name):
    z = semi()
    return {k: z[f"{name}/{k}"] for k in FIELDS}


ELL_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "elliptic.npz")
_ze = None


def ell():
    """tests/golden/elliptic.npz (make_elliptic_golden.py): the elliptic-closed solver."""
    global _ze
    if _ze is None:
        _ze = dict(np.load(ELL_PATH))
    return _ze


def ell_cases():
    return json.loads(bytes(ell()["meta_json"]).decode())


def ell_desc(name):
    return abi.frame_desc(**ell_cases()[name])


def ell_result(name):
    z = ell()
    return {k: z[f"{name}/{k}"] for k in FIELDS}
