import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def built():
    """Library and oracle built in-tree (no-op when up to date)."""
    from fdv_b200 import build as fb
    from oracle import build as ob
    fb.build()
    ob.build_all()
    return True


def scene_frames(kw):
    """Frames of a golden case's scene: the moving-rectangle generator, or
    the camera-like stress generator when kind is "camera"."""
    import fdv_b200 as F
    kw = dict(kw)
    n = kw.pop("nframes")
    w, h = kw.pop("w"), kw.pop("h")
    if kw.pop("kind", "rects") == "camera":
        return F.CamScene(w, h, n, **kw).frames(n)
    return F.Scene(w, h, n, **kw).frames(n)
