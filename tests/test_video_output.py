"""Video output (3di_b200/video.py): the reference's scale list, per-frame averages, NaN rows
for frames without a reconstruction and the text layout of .expressions / .poses / .illums
(video_fitter.cu:271-280, 355-393, 2603-2830; funcs.h:112-124), and the multi-scale batch
against one fit per scale."""
import importlib

import numpy as np
import pytest

video = importlib.import_module("3di_b200.video")
F32 = np.float32


def test_ref_sizes_follow_the_reference_list():
    assert [float(v) for v in video.ref_sizes(86.0, 4)] == [86.0, 96.0, 94.0, 100.0]
    s15 = video.ref_sizes(86.0, 15)
    assert [float(v) for v in s15[8:]] == [93.5, 91.5, 97.5, 95.5, 79.5, 82.5, 85.5]
    s17 = video.ref_sizes(86.0, 17)       # std::vector::resize pads with zeros
    assert float(s17[15]) == 0.0 and float(s17[16]) == 0.0


def test_rotation_matches_the_oracle(O):
    rng = np.random.default_rng(4)
    for _ in range(20):
        u = rng.normal(0, 0.4, 3).astype(F32)
        R = video.rotation_matrix(u)
        Ro, _ = O.rotation(u)
        assert np.array_equal(Ro.view(np.uint32), R.view(np.uint32))


def test_euler_angles_of_axis_rotations():
    for ang in (0.1, -0.3, 0.7):
        # rotation about the optical (z) axis: roll only
        yaw, pitch, roll = video.euler_angles(video.rotation_matrix([0.0, 0.0, ang]))
        assert abs(float(roll) - ang) < 1e-6 and abs(float(yaw)) < 1e-6 and abs(float(pitch)) < 1e-6


def test_averages_nan_rows_and_text_layout(tmp_path):
    out = video.VideoOutput(K=3, nres=2)
    out.add_exp_coeffs(0, [1.0, 2.0, 3.0])
    out.add_exp_coeffs(0, [3.0, 4.0, 5.0])
    out.add_exp_coeffs(2, [0.1, 0.2, 0.3])
    for fid, u in ((0, 0.1), (0, 0.3), (2, 0.2)):
        out.add_pose(fid, [1.0, 2.0, 3.0, 0.0, 0.0, u])
    out.add_illum(0, [0.5, 0.6, 0.7, 1.0])
    out.add_illum(0, [9.0, 9.0, 9.0, 9.0])       # only the first illumination of a frame stays
    out.add_illum(2, [0.1, 0.2, 0.3, 1.0])
    avg0 = out.compute_avg_exp_coeffs(0)
    assert np.array_equal(avg0, np.array([F32(1) / F32(2) + F32(3) / F32(2), 3.0, 4.0], F32))
    assert np.array_equal(out.compute_avg_exp_coeffs(0, ignore_first=True), np.array([3, 4, 5], F32))
    assert np.isnan(out.compute_avg_exp_coeffs(1)).all()                       # no reconstruction
    assert np.array_equal(out.combine_exp_coeffs(2)[:3], np.array([0.1, 0.2, 0.3], F32))
    assert np.isnan(out.combine_exp_coeffs(2)[3:]).all()
    assert np.array_equal(out.get_illum(0), np.array([0.5, 0.6, 0.7, 1.0], F32))
    out.save_expressions(str(tmp_path / "a.expressions"))
    out.save_expressions_all(str(tmp_path / "a.all"))
    out.save_poses(str(tmp_path / "a.poses"))
    out.save_illums(str(tmp_path / "a.illums"))
    lines = (tmp_path / "a.expressions").read_text().split("\n")
    # frames 0 .. max id - 1 (the reference stops before the largest id), each value '%.7g '
    assert lines == ["2 3 4 ", "nan nan nan ", ""]
    assert (tmp_path / "a.all").read_text().split("\n")[2].startswith("0.1 0.2 0.3 nan nan nan ")
    pl = (tmp_path / "a.poses").read_text().split("\n")
    vals = [float(v) for v in pl[0].split()]
    assert len(vals) == 9 and vals[:5] == [1.0, 2.0, 3.0, 0.0, 0.0] and abs(vals[5] - 0.2) < 1e-7
    assert abs(vals[8] - 0.2) < 1e-6                                   # roll of a z rotation
    assert pl[1].split() == ["nan"] * 9
    assert (tmp_path / "a.illums").read_text().split("\n")[0] == "0.5 0.6 0.7 1 "


def test_seven_significant_digits():
    assert "%.7g " % float(F32(1.0 / 3.0)) == "0.3333333 "
    assert "%.7g " % float(F32(1e-8)) == "1e-08 "


@pytest.mark.gpu
def test_multiscale_batch_equals_one_fit_per_scale(tdi, synth):
    import os
    tdi.require_gpu()
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "preprocess_golden.npz"))
    m = synth.make_model(5000, 9800, 0)
    model = tdi.Model(m)
    K = m.n_expr
    bgr, xp, yp, fs, cam = z["bgr0"], z["xp0"], z["yp0"], z["face_size0"], z["cam0"]
    T = 2
    bgr2 = np.stack([bgr, bgr[:, ::-1].copy()])
    xp2, yp2 = np.stack([xp, xp]), np.stack([yp, yp])
    fs2, cam2 = np.array([fs, fs], F32), np.stack([cam, cam])
    bounds = np.tile(np.array([-0.2, -0.2, 0.2, 0.2], F32)[None, :, None], (T, 1, 51))
    x0 = np.zeros((T, K + 6), F32)
    x0[:, K + 2] = 1.0
    lam0 = np.tile(synth.LAMBDA_INIT, (T, 1)).astype(F32)
    L = np.full(T, synth.L_INTENSITY, F32)
    cfg = tdi.default_config(max_iters_rigid=3)
    sizes = video.ref_sizes(86.0, 3)
    out = video.VideoOutput(K, nres=3)
    video.fit_multiscale(tdi.Batch(model, len(sizes) * T), bgr2, xp2, yp2, bounds, fs2, cam2, x0, lam0, L,
                         cfg, sizes, [5, 6], out)
    single = tdi.Batch(model, T)
    for s, ref in enumerate(sizes):
        single.set_video_frames(bgr2, xp2, yp2, bounds, fs2, cam2, float(ref))
        single.set_state(x0, lam0, L)
        single.fit(cfg)
        x, lam, rep = single.get_state()
        for t, fid in enumerate([5, 6]):
            assert np.array_equal(out.exp_coefs[fid][s].view(np.uint32), x[t, :K].view(np.uint32))
            assert np.array_equal(out.poses[fid][s].view(np.uint32), x[t, K:K + 6].view(np.uint32))
    assert all(len(out.exp_coefs[fid]) == len(sizes) for fid in (5, 6))
