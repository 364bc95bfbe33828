"""Frame preprocessing (tdi_batch_set_video_frames): the oracle restatement against golden
crops made with OpenCV (tests/golden/make_preprocess_golden.py), and the device path against
both. The reference forms its crops with OpenCV on the host (input_data.cu:43-53,
video_fitter.cu:537-550); this build forms them on the GPU."""
import os

import numpy as np
import pytest

import preprocess as P

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "preprocess_golden.npz")


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def _case(z, k):
    return (z[f"bgr{k}"], z[f"xp{k}"], z[f"yp{k}"], z[f"face_size{k}"], z[f"cam{k}"], z["ref_face_size"])


def test_oracle_matches_opencv_golden_crops(golden):
    for k in range(int(golden["n_cases"])):
        crop, xl, yl, cam, fs, x0, y0 = P.video_frame(*_case(golden, k))
        assert (x0, y0) == tuple(int(v) for v in golden[f"x0y0_{k}"])
        assert np.array_equal(_bits(crop), _bits(golden[f"crop{k}"])), k


def test_gray_formula_on_every_color():
    # BGR2GRAY on 8-bit data: the weights of OpenCV 4 (checked against cv2 exhaustively when
    # the golden file was made); here the formula's range and the black/white end points
    b = np.array([[[0, 0, 0], [255, 255, 255], [255, 0, 0], [0, 255, 0], [0, 0, 255]]], np.uint8)
    g = P.gray(b)
    y8 = np.rint(g[0] * 255).astype(int)
    assert list(y8) == [0, 255, 29, 150, 76]


def test_resize_identity_and_border_columns():
    rng = np.random.default_rng(3)
    img = rng.random((7, 9)).astype(np.float32)
    assert np.array_equal(P.resize_linear(img, 1.0), img)   # unit scale: taps (1, 0)
    up = P.resize_linear(img, 2.0)
    assert up.shape == (14, 18)
    # output columns at or past the last source column take that column alone
    assert np.array_equal(up[:, -1], P.resize_linear(img[:, -1:], 2.0)[:, 0])
    s, a0, a1, single = P.resize_row_coords(9, 18, 0.5)
    assert single[-1] and s[-1] == 8 and a1[-1] == 0


@pytest.mark.gpu
def test_device_crops_match_golden_and_oracle(tdi, synth, golden):
    tdi.require_gpu()
    m = synth.make_model(5000, 9800, 0)
    model = tdi.Model(m)
    batch = tdi.Batch(model, 8)
    bounds = np.zeros((1, 4, 51), np.float32)
    for k in range(int(golden["n_cases"])):
        bgr, xp, yp, fs, cam, ref = _case(golden, k)
        batch.set_video_frames(bgr[None], xp[None], yp[None], bounds, [fs], cam[None], float(ref))
        crop = batch.read(0, tdi.READ_CROP)
        assert np.array_equal(_bits(crop), _bits(golden[f"crop{k}"])), k
        o_crop, xl, yl, ocam, ofs, x0, y0 = P.video_frame(bgr, xp, yp, fs, cam, ref)
        fd = batch.read(0, tdi.READ_FRAME_DATA)
        assert np.array_equal(_bits(fd["xl"]), _bits(xl)) and np.array_equal(_bits(fd["yl"]), _bits(yl))
        assert np.array_equal(_bits(fd["cam"]), _bits(ocam))
        assert np.float32(fd["face_size"]) == ofs and (fd["x0"], fd["y0"]) == (x0, y0)
    # several frames in one call: one image at different face sizes
    bgr, xp, yp, fs, cam, ref = _case(golden, 0)
    sizes = np.array([fs, 0.8 * fs, 1.7 * fs, 3.0 * fs, 0.4 * fs], np.float32)
    n = len(sizes)
    batch.set_video_frames(np.repeat(bgr[None], n, 0), np.repeat(xp[None], n, 0), np.repeat(yp[None], n, 0),
                           np.zeros((n, 4, 51), np.float32), sizes, np.repeat(cam[None], n, 0), float(ref))
    for f in range(n):
        o_crop = P.video_frame(bgr, xp, yp, sizes[f], cam, ref)[0]
        assert np.array_equal(_bits(batch.read(f, tdi.READ_CROP)), _bits(o_crop)), f
