"""Shared fixtures. The CPU oracle (oracle/) is the checker; the product is 3di_b200/."""
import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def tdi():
    return importlib.import_module("3di_b200")


@pytest.fixture(scope="session")
def synth():
    return importlib.import_module("3di_b200.synth")


@pytest.fixture(scope="session")
def O():
    import oracle
    oracle.build()
    return oracle


def make_case(synth, O, n_vertices, n_triangles, config_id, n_frames, frames_kw, noise=0.02,
              surface="face"):
    """Model, frames with noisy targets rendered by the oracle at the true states."""
    m = synth.make_model(n_vertices, n_triangles, config_id, surface=surface)
    fr = synth.make_frames(m, n_frames, config_id, **frames_kw)
    om = O.Model(m)
    cfg = O.config()
    tg = []
    for i in range(n_frames):
        img, n, fl = O.render_target(om, fr, i, cfg, fr.state_true[i], fr.lam_true[i],
                                     synth.L_INTENSITY)
        tg.append(img)
    fr.target = synth.add_noise(np.stack(tg), noise, config_id)
    return m, fr, om


@pytest.fixture(scope="session")
def small_case(synth, O):
    """5,000 vertices / 9,800 triangles, 256x256 frames (the reference's plain single-frame case)."""
    return make_case(synth, O, 5000, 9800, 0, 3, dict(image_wh=(256, 256), tz=0.6))


@pytest.fixture(scope="session")
def full_case(synth, O):
    """53,490 vertices / 106,466 triangles, 1080p frames rescaled to the 256x256 crop."""
    return make_case(synth, O, 53490, 106466, 1, 2, dict(image_wh=(1920, 1080), box_range=(300, 600)))


@pytest.fixture(scope="session")
def rough_case(synth, O):
    """The full-size model with rough bases: the mesh folds over itself, so most pixels are
    covered by several triangles (depth tests, ties and dropped fragments everywhere)."""
    return make_case(synth, O, 53490, 106466, 1, 2, dict(image_wh=(1920, 1080), box_range=(300, 600)),
                     surface="rough")
