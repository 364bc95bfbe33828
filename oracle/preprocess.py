"""CPU restatement of the reference's frame preprocessing. TEST INFRASTRUCTURE ONLY.

Only tests/ use this module, as the checker of tdi_batch_set_video_frames. It restates, in
numpy float32 arithmetic (one rounding per operation, no fused multiply-add):

* InputData::get_resized_frame (src/lib/input_data.cu:43-53): cv::cvtColor(BGR2GRAY) on
  8-bit pixels, convertTo(CV_32F) and division by 255, cv::resize(INTER_LINEAR) by the
  frame's resize coefficient, cv::copyMakeBorder with DIMX/DIMY zero columns/rows;
* the crop of VideoFitter::fit_to_video_frame (src/lib/video_fitter.cu:537-550): the 256x256
  rectangle at the crop origin, transposed (stored x-major);
* InputData::get_resized_landmarks (input_data.cu:32-40), Camera::update_camera
  (camera.h:162-174) with resize coefficient ref_face_size / face_size
  (video_fitter.cu:359, 402), Renderer::set_x0_short_y0_short with padding
  (renderer.cu:580-598) and the face size of funcs.cu:44-54.

The OpenCV steps follow OpenCV 4 (the reference's dependency; pinned against opencv-python
4.13.0 by tests/golden/make_preprocess_golden.py): BGR2GRAY on 8-bit data is
(3735 B + 19235 G + 9798 R + 2^14) >> 15; convertTo with scale 1/255 multiplies by the float
(1/255.); INTER_LINEAR on float images is OpenCV's generic resize (the path taken when
OpenCV runs without Intel IPP, cv2.ipp.setUseIPP(False)): source coordinate
(float)((X + 0.5) / c - 0.5) in double arithmetic, weights 1 - f and f as floats, clamped
columns as described in resize_row_coords, clamped row indices with unchanged weights, each
pass two float products and a float sum.
"""
from __future__ import annotations

import numpy as np

NL, DIM = 51, 256
F32 = np.float32


def gray(bgr: np.ndarray) -> np.ndarray:
    """8-bit BGR [H][W][3] -> float32 gray [H][W] (cvtColor BGR2GRAY, then / 255)."""
    b = bgr[..., 0].astype(np.int64)
    g = bgr[..., 1].astype(np.int64)
    r = bgr[..., 2].astype(np.int64)
    y8 = (b * 3735 + g * 19235 + r * 9798 + 16384) >> 15
    return y8.astype(F32) * F32(1.0 / 255.0)


def resize_row_coords(n_src: int, n_dst: int, inv: float):
    """Column taps of cv::resize INTER_LINEAR: (index, weight0, weight1, single) per output.
    A coordinate left of the image takes index 0 with weights (1, 0); one at or past the
    last column takes that column alone."""
    X = np.arange(n_dst, dtype=np.float64)
    f = ((X + 0.5) * inv - 0.5).astype(F32)
    s = np.floor(f).astype(np.int64)
    f = (f - s.astype(F32)).astype(F32)
    left = s < 0
    f[left] = F32(0)
    s[left] = 0
    single = s + 1 >= n_src
    f[single] = F32(0)
    s[single] = n_src - 1
    return s, (F32(1) - f).astype(F32), f, single


def resize_linear(src: np.ndarray, coef: float) -> np.ndarray:
    """cv::resize(src, Size(), coef, coef, INTER_LINEAR) of a float32 image (generic path)."""
    H, W = src.shape
    c = float(np.float32(coef))
    rw, rh = int(np.rint(W * c)), int(np.rint(H * c))
    inv = 1.0 / c
    sx, a0, a1, single = resize_row_coords(W, rw, inv)
    sx1 = np.where(single, sx, sx + 1)
    # horizontal pass on every source row
    t0 = (src[:, sx] * a0).astype(F32)
    t1 = (src[:, sx1] * a1).astype(F32)
    h = np.where(single[None, :], src[:, sx], (t0 + t1).astype(F32)).astype(F32)
    # vertical pass: row indices clamped, weights unchanged
    Y = np.arange(rh, dtype=np.float64)
    fy = ((Y + 0.5) * inv - 0.5).astype(F32)
    sy = np.floor(fy).astype(np.int64)
    fy = (fy - sy.astype(F32)).astype(F32)
    b0, b1 = (F32(1) - fy).astype(F32), fy
    r0 = np.clip(sy, 0, H - 1)
    r1 = np.clip(sy + 1, 0, H - 1)
    u0 = (h[r0, :] * b0[:, None]).astype(F32)
    u1 = (h[r1, :] * b1[:, None]).astype(F32)
    return (u0 + u1).astype(F32)


def crop_origin(xl, yl):
    """(ushort) max(min - size / 1.5, 0) per axis, the subtraction in double."""
    xl = np.asarray(xl, F32)
    yl = np.asarray(yl, F32)
    sz = F32(max(F32(xl.max() - xl.min()), F32(yl.max() - yl.min())))
    x0 = F32(float(xl.min()) - float(sz) / 1.5)
    y0 = F32(float(yl.min()) - float(sz) / 1.5)
    return int(max(x0, F32(0))) & 0xFFFF, int(max(y0, F32(0))) & 0xFFFF


def face_size(xl, yl):
    xl = np.asarray(xl, F32)
    yl = np.asarray(yl, F32)
    return F32(max(F32(xl.max() - xl.min()), F32(yl.max() - yl.min())))


def video_frame(bgr, xp, yp, face_sz, cam, ref_face_size):
    """One frame: (crop [65536] x-major, xl, yl, cam [4], face size, x0, y0)."""
    c = F32(F32(ref_face_size) / F32(face_sz))
    xl = (c * np.asarray(xp, F32)).astype(F32)
    yl = (c * np.asarray(yp, F32)).astype(F32)
    cm = (np.asarray(cam, F32) * c).astype(F32)
    x0, y0 = crop_origin(xl, yl)
    img = resize_linear(gray(np.asarray(bgr, np.uint8)), float(c))
    rh, rw = img.shape
    pad = np.zeros((rh + DIM, rw + DIM), F32)     # copyMakeBorder: DIMY rows, DIMX columns
    pad[:rh, :rw] = img
    big = np.zeros((y0 + DIM, x0 + DIM), F32)     # (origins past the padded image read zeros)
    hh, ww = min(pad.shape[0], big.shape[0]), min(pad.shape[1], big.shape[1])
    big[:hh, :ww] = pad[:hh, :ww]
    crop = big[y0:y0 + DIM, x0:x0 + DIM]          # [y][x]
    return np.ascontiguousarray(crop.T).reshape(-1), xl, yl, cm, face_size(xl, yl), x0, y0
