"""Orthographic pose initialisation (tdi_orthographic_init; the reference's
OrthographicInitializer::fit_model, orthographic_initializer.cu:243-380): the oracle
recovers known scaled-orthographic poses, and the device fit equals the oracle bit for bit
(state, last trial rotation, iterations) with the Euler angles formed from that rotation."""
import importlib
import math

import numpy as np
import pytest

F32 = np.float32


def _landmarks(O, p0L, rng, n, unit_m):
    """Scaled orthographic projections of the landmark points at random poses, with noise:
    600-1200 px per metre, offsets of about 1 cm (the model is in units of ``unit_m`` metres)."""
    xl, yl, us = [], [], []
    for _ in range(n):
        u = rng.normal(0, 0.15, 3).astype(F32)
        R, _ = O.rotation(u)
        rp = R.reshape(3, 3, order="F").astype(np.float64) @ p0L.astype(np.float64)
        s = rng.uniform(600, 1200) * unit_m
        xl.append((s * (rp[0] + rng.normal(0, 0.01) / unit_m) + 400 + rng.normal(0, 0.5, 51)).astype(F32))
        yl.append((s * (rp[1] + rng.normal(0, 0.01) / unit_m) + 300 + rng.normal(0, 0.5, 51)).astype(F32))
        us.append(u)
    return np.array(xl), np.array(yl), np.array(us)


@pytest.fixture(scope="module")
def p0L(synth):
    m = synth.make_model(5000, 9800, 0)
    return np.ascontiguousarray(m.mean[:, m.lis].astype(F32))


def _degrees(R):
    video = importlib.import_module("3di_b200.video")
    return [F32(float(F32(a * F32(180.0))) / math.pi) for a in video.euler_angles(R)]


def test_oracle_fits_scaled_orthographic_landmarks(O, synth, p0L):
    rng = np.random.default_rng(7)
    xl, yl, _ = _landmarks(O, p0L, rng, 12, synth.UNIT_M)
    fitted, rmss = 0, []
    for f in range(12):
        x, R, q = O.orthographic(xl[f], yl[f], p0L.reshape(-1))
        assert 1 <= q <= 100
        if q == 1:
            continue                 # the first line search failed: the start point stays
        fitted += 1
        Rx, _ = O.rotation(x[4:])
        rp = Rx.reshape(3, 3, order="F").astype(np.float64) @ p0L.astype(np.float64)
        ex = x[2] * (rp[0] + x[0]) - (xl[f] - xl[f].mean())
        ey = x[3] * (rp[1] + x[1]) - (yl[f] - yl[f].mean())
        rmss.append(math.sqrt(float(np.mean(np.concatenate([ex, ey]) ** 2))))
    assert fitted >= 8, fitted
    # landmark noise is 0.5 px; the line search can stop early on a pose, as the reference's does
    assert np.median(rmss) < 1.5 and max(rmss) < 10.0, rmss


@pytest.mark.gpu
def test_device_matches_oracle(tdi, O, synth, p0L):
    tdi.require_gpu()
    rng = np.random.default_rng(11)
    xl, yl, _ = _landmarks(O, p0L, rng, 37, synth.UNIT_M)
    x, ypr, it = tdi.orthographic_init(xl, yl, p0L)
    for f in range(37):
        ox, oR, oq = O.orthographic(xl[f], yl[f], p0L.reshape(-1))
        assert it[f] == oq
        assert np.array_equal(x[f].view(np.uint32), ox.view(np.uint32)), f
        assert np.array_equal(ypr[f].view(np.uint32), np.array(_degrees(oR), F32).view(np.uint32)), f
