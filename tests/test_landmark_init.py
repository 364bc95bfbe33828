"""Landmark initialisation (tdi_batch_landmark_init; the reference's
Logbarrier_Initializer::initialize_with_orthographic_t, set_minimal_slack and fit_model with a
slack variable, logbarrier_initializer.cu:1041-1269,1862-1918): the oracle's restatement on
CPU, and the device path against it bit for bit -- success, Newton iterations, slack and the
state handed to the image fit -- including frames whose orthographic fit ends mirrored."""
import numpy as np
import pytest


def _p0L(m):
    return np.ascontiguousarray(m.mean[:, m.lis].astype(np.float32))


def _mirrored(fr):
    """The frames' landmarks reflected about their centre column: the orthographic fit then
    converges to a mirrored pose (sigma_x < 0)."""
    import copy
    g = copy.deepcopy(fr)
    c = fr.xl.mean(axis=1, keepdims=True)
    g.xl = (2 * c - fr.xl).astype(np.float32)
    return g


def test_oracle_reaches_feasible_landmark_boxes(O, small_case):
    """Frames the method reports as successful end with every landmark inside its box."""
    m, fr, om = small_case
    fs = O.FrameSet(fr)
    K = m.n_expr
    ok_any = False
    for i in range(fr.n_frames):
        x, slack, ok, it, flip = O.landmark_init(om, fs, i, _p0L(m))
        assert it >= 1
        if not ok:
            continue
        ok_any = True
        assert slack < -0.01
        geo, _ = O.vertex_stage(om, x, fr.cam[i])
        xp, yp = geo[6][m.lis], geo[7][m.lis]
        b, fsz = fr.bounds[i], fr.face_size[i]
        assert np.all(xp >= fr.xl[i] + b[0] * fsz) and np.all(xp <= fr.xl[i] + b[2] * fsz)
        assert np.all(yp >= fr.yl[i] + b[1] * fsz) and np.all(yp <= fr.yl[i] + b[3] * fsz)
    assert ok_any


def test_oracle_refits_mirrored_orthographic_solutions(O, small_case):
    m, fr, om = small_case
    g = _mirrored(fr)
    fs = O.FrameSet(g)
    flips = [O.landmark_init(om, fs, i, _p0L(m))[4] for i in range(g.n_frames)]
    assert any(flips)


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.mark.gpu
@pytest.mark.parametrize("case_name", ["small_case", "full_case", "mirrored"])
def test_device_matches_oracle(request, tdi, synth, O, case_name):
    tdi.require_gpu()
    m, fr, om = request.getfixturevalue("small_case" if case_name == "mirrored" else case_name)
    if case_name == "mirrored":
        fr = _mirrored(fr)
    model = tdi.Model(m)
    batch = tdi.Batch(model, fr.n_frames)
    batch.set_frames(fr)
    ok, slack, it = batch.landmark_init(_p0L(m))
    lam = np.tile(synth.LAMBDA_INIT, (fr.n_frames, 1))
    L = np.full(fr.n_frames, synth.L_INTENSITY, np.float32)
    batch.set_state(None, lam, L)
    x, _, _ = batch.get_state()
    fs = O.FrameSet(fr)
    for i in range(fr.n_frames):
        ox, oslack, ook, oit, oflip = O.landmark_init(om, fs, i, _p0L(m))
        assert ok[i] == ook and it[i] == oit, (i, ok[i], ook, it[i], oit)
        assert _bits(slack[i]) == _bits(np.float32(oslack)), i
        assert np.array_equal(_bits(x[i]), _bits(ox)), i


@pytest.mark.gpu
def test_initialised_fit_matches_oracle(tdi, synth, O, small_case):
    """Landmark initialisation then the image fit, all on the device, against the oracle doing
    the same: the fits start from identical states and follow the same iterates."""
    tdi.require_gpu()
    m, fr, om = small_case
    model = tdi.Model(m)
    batch = tdi.Batch(model, fr.n_frames)
    batch.set_frames(fr)
    ok, slack, it = batch.landmark_init(_p0L(m))
    lam = np.tile(synth.LAMBDA_INIT, (fr.n_frames, 1))
    L = np.full(fr.n_frames, synth.L_INTENSITY, np.float32)
    batch.set_state(None, lam, L)
    batch.fit(tdi.default_config(max_iters_rigid=10))
    x, lamf, rep = batch.get_state()
    fs = O.FrameSet(fr)
    x0 = np.stack([O.landmark_init(om, fs, i, _p0L(m))[0] for i in range(fr.n_frames)])
    ox, olam, orep = O.fit_frames(om, fs, O.config(max_iters_rigid=10), x0, lam, L)
    for i in range(fr.n_frames):
        assert rep[i].flags == orep[i].flags and rep[i].iters_rigid == orep[i].iters_rigid
        err = np.abs(x[i] - ox[i]) / np.maximum(np.abs(ox[i]), 1e-2)
        assert err.max() <= 1e-5, err.max()
