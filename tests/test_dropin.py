"""The drop-in video_from_saved_identity (3di_b200/video_from_saved_identity.py): the
reference's file formats written from the synthetic model and read back (CPU), and the whole
command on a short synthetic video (GPU)."""
import importlib
import os

import numpy as np
import pytest

F32 = np.float32


def _write_model(root, m, MM="SYNTH-5000"):
    """The model in the reference's files: models/MMs/<MM>/ (prepare_BFM.py:280-307 layouts),
    the identity .shp/.tex files, a YAML configuration."""
    d = os.path.join(root, "models", "MMs", MM)
    os.makedirs(os.path.join(d, "E"), exist_ok=True)
    for c, name in enumerate(("EX_79", "EY_79", "EZ_79")):
        np.savetxt(os.path.join(d, "E", name + ".dat"), m.E[:, c, :].astype(np.float64))
    np.savetxt(os.path.join(d, "tl.dat"), m.tl.T + 1, fmt="%d")
    np.savetxt(os.path.join(d, "li.dat"), m.lis, fmt="%d")
    np.savetxt(os.path.join(d, "p0L_mat.dat"), m.mean[:, m.lis].T.astype(np.float64))
    np.savetxt(os.path.join(d, "E", "sigma_epsilons_79_lowerv2.dat"), (m.eps_lb / F32(1.75)).astype(np.float64))
    np.savetxt(os.path.join(d, "E", "sigma_epsilons_79_upperv2.dat"), (m.eps_ub / F32(1.75)).astype(np.float64))
    shp = os.path.join(root, "id.shp")
    tex = os.path.join(root, "id.tex")
    np.savetxt(shp, m.mean.T.astype(np.float64))
    np.savetxt(tex, m.tex[:, None].astype(np.float64))
    cfg = os.path.join(root, "cfg.yaml")
    with open(cfg, "w") as fh:
        fh.write('%YAML:1.0\n---\nEXP_BASIS: "GLOBAL79"\nOPTS_DELTA_EPS: 1.75\nREF_FACE_SIZE: 78\n'
                 f"KERNEL_SIGMA: 0.75\nNRES_COEFS: 2\nMM: {MM}\nTWOSTAGE_ILLUM: 0\nFINETUNE_EXPRESSIONS: 0\n")
    return cfg, shp, tex


def test_reference_files_read_back(tmp_path, synth):
    vfsi = importlib.import_module("3di_b200.video_from_saved_identity")
    m = synth.make_model(5000, 9800, 0)
    cfg_path, shp, tex = _write_model(str(tmp_path), m)
    cfg = vfsi.read_config(cfg_path)
    assert cfg["MM"] == "SYNTH-5000" and cfg["NRES_COEFS"] == 2 and cfg["REF_FACE_SIZE"] == 78.0
    assert cfg["FINETUNE_COEF"] == 1.5 and cfg["NITERS_SUCCESS"] == 6      # the reference's defaults
    m2, p0L = vfsi.read_model(os.path.join(str(tmp_path), "models", "MMs", cfg["MM"]), cfg, shp, tex)
    assert np.array_equal(m2.E, m.E) and np.array_equal(m2.mean, m.mean) and np.array_equal(m2.tex, m.tex)
    assert np.array_equal(m2.tl, m.tl) and np.array_equal(m2.lis, m.lis)
    assert np.array_equal(p0L, m.mean[:, m.lis])
    np.testing.assert_allclose(m2.eps_ub, m.eps_ub, rtol=1e-6)
    np.testing.assert_allclose(m2.eps_ub_ft, m.eps_ub * F32(1.5), rtol=1e-6)


def test_landmarks_camera_and_boxes(tmp_path):
    vfsi = importlib.import_module("3di_b200.video_from_saved_identity")
    rng = np.random.default_rng(3)
    xy = rng.uniform(100, 200, (5, 102))
    p = os.path.join(str(tmp_path), "lmks.txt")
    np.savetxt(p, xy)
    xp, yp = vfsi.read_landmarks(p)
    assert xp.shape == (5, 51) and np.array_equal(xp, xy[:, 0::2].astype(F32)) and np.array_equal(yp, xy[:, 1::2].astype(F32))
    fs = vfsi.face_size(xp[0], yp[0])
    assert fs == max(int(xp[0].max()) - int(xp[0].min()), int(yp[0].max()) - int(yp[0].min()))
    cam = vfsi.camera("40", 1920, 1080)
    assert cam[2] == 960 and cam[3] == 540
    np.testing.assert_allclose(cam[0], 960 / np.tan(np.radians(20)), rtol=1e-6)
    b = vfsi.constant_bounds(2)
    assert b.shape == (2, 4, 51) and np.all(b[:, 0] < -0.08) and np.all(b[:, 2] > 0.08)


def _write_video(root, tdi, synth, O, m, n=4):
    """A short video of the synthetic subject (small head rotations) rendered by the library at
    the crop scale, pasted into 400x300 frames; landmarks of the true states with 0.5 px noise."""
    import cv2
    fr = synth.make_frames(m, n, 0, image_wh=(400, 300), tz=0.75)
    K = m.n_expr
    rng = np.random.default_rng(5)
    fr.state_true[:, K + 3:] = rng.uniform(-0.12, 0.12, (n, 3)).astype(F32)
    fr.state_true[:, :K] *= F32(0.3)
    model = tdi.Model(m)
    batch = tdi.Batch(model, n)
    fr.target = np.zeros((n, 65536), F32)
    # landmarks and crop origins of the true states in 400x300 frames (no rescaling: c = 1)
    geo = []
    om = O.Model(m)
    for i in range(n):
        g, _ = O.vertex_stage(om, fr.state_true[i], fr.cam[i])
        geo.append(g)
        fr.xl[i] = g[6][m.lis] + rng.normal(0, 0.5, 51).astype(F32)
        fr.yl[i] = g[7][m.lis] + rng.normal(0, 0.5, 51).astype(F32)
        fr.x0y0[i] = 0
    batch.set_frames(fr)
    batch.set_state(fr.state_true, fr.lam_true, np.full(n, synth.L_INTENSITY, F32))
    img, _ = batch.render()
    path = os.path.join(root, "v.avi")
    w = cv2.VideoWriter(path, cv2.VideoWriter_fourcc(*"MJPG"), 24, (400, 300))
    for i in range(n):
        crop = img[i].reshape(256, 256).T                     # x-major -> rows are y
        frame = np.zeros((300, 400), F32)
        frame[:256, :256] = crop
        w.write(cv2.cvtColor(np.clip(frame * 255, 0, 255).astype(np.uint8), cv2.COLOR_GRAY2BGR))
    w.release()
    lm = os.path.join(root, "lmks.txt")
    np.savetxt(lm, np.stack([np.stack([fr.xl[i], fr.yl[i]], 1).reshape(-1) for i in range(n)]))
    fov = np.degrees(2 * np.arctan(200.0 / fr.cam[0][0]))
    return path, lm, f"{fov:.6f}", fr


@pytest.mark.gpu
def test_dropin_runs_end_to_end(tmp_path, tdi, synth, O):
    tdi.require_gpu()
    vfsi = importlib.import_module("3di_b200.video_from_saved_identity")
    m = synth.make_model(5000, 9800, 0)
    root = str(tmp_path)
    cfg, shp, tex = _write_model(root, m)
    video, lm, fov, fr = _write_video(root, tdi, synth, O, m)
    outs = [os.path.join(root, f"o.{e}") for e in ("expressions", "poses", "illums")]
    assert vfsi.main([video, lm, cfg, fov, shp, tex, *outs, "--models-root", root]) == 0
    rows = [np.loadtxt(p, ndmin=2) for p in outs]
    n, r = fr.n_frames, rows[1].shape[0]
    # frames 0 .. (last frame with a reconstruction) - 1, as the reference writes them
    assert 1 <= r <= n - 1
    assert rows[0].shape == (r, 79) and rows[1].shape == (r, 9) and rows[2].shape == (r, 4)
    ok = ~np.isnan(rows[1][:, 0])
    assert ok.sum() >= 1
    K = m.n_expr
    tz_true = fr.state_true[:r, K + 2]
    assert np.all(np.abs(rows[1][ok, 2] - tz_true[ok]) <= 0.25 * tz_true[ok]), (rows[1][ok, 2], tz_true[ok])
    with open(outs[1]) as fh:
        first = fh.readline()
    assert first.endswith(" \n") and len(first.split()) == 9
